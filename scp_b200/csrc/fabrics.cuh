// fabrics.cuh -- the gauged stepper with three matter fabrics C, Q, L under
// one shared compact U(1) (the reference's multi-fabric model: per-fabric
// force force_fabric_gauged_accum and its driver compute_forces_complex_
// gauge_mf, sfa/sim/scp_sim.c:1274-1433; the EM charge density em_rho_at,
// :184-197; per-fabric charges compute_mf_charges, :2247-2261).
//
// Physics.  Every fabric is a complex Cosserat multiplet with its own bag
// potential, transported by the charge-q_f links e^{i q_f th}; the field
// kick is the plaquette term plus sum_f g q_f J_f, and the Gauss law uses
// rho_em = sum_f q_f rho_f.  With the C-Q lock Q equals C at every step: the
// reference copies C into Q after each force and kick, so C moves under the
// q_Q force (the Q pass overwrites C's accelerations) while both fabrics add
// their currents, g q_C J_C(C) + g q_Q J_Q(C).  Here Q's arrays are C's.
//
// Structure.  One time step is one ring launch per fabric and one for the
// links.  A fabric launch stages the fabric's 12 matter fields and the three
// link angles, advances the fabric's matter by the fused leapfrog, and adds
// its currents g q J to a per-site accumulator; the link launch stages the
// angles, forms the plaquette term, and kicks E and drifts the angles with
// the accumulated currents.  Positions (two alternating buffers) and momenta
// hold C with the links (15 arrays, the fused step's order), then L (12),
// then Q (12) when it is not locked.
#pragma once
#include "multiplet.cuh"
#include "ring.cuh"

namespace scp {

struct FabConsts {
    int N;
    long long N3;
    double L, dx, dV, idx1, idx2, inva, hdt, dt;
    double mu, kappa, m2, mtheta2, eta;
    double g, stp, gad;
    double damp_width, damp_rate;
};

// One fabric's matter step.  The force uses links of charge qf; the current
// g qf J(qf) goes to the accumulator, preceded, with SECOND, by g qx J(qx)
// over the same fields (the locked pair's C current).
template <bool SECOND>
struct FabricPass {
    static constexpr int TH = 12;
    static constexpr int NR = 15;
    static constexpr int MIN_CTAS = 1;

    struct Args {
        RingSrc<NR> src;      // this fabric's 12 matter positions, then th
        int N;
        FabConsts c;
        double qf, gqf;       // force charge, current weight g qf
        double qx, gqx;       // second current (SECOND)
        const double *win;    // 12 momenta: w_n (v_0 on the first launch)
        double *wout, *xout, *sout;
        double *kacc;         // 3 arrays: accumulated currents
        int *flag;
        int first, sync, damp, accumulate;
    };

    struct Carry {
        double cm, sm;        // charge-qf link phase along i at x - i
        double cmx, smx;      // the same for qx
    };

    __device__ static void prefetch(const Args &A, long long idx) {
#pragma unroll
        for (int f = 0; f < 12; f++) prefetch_l2(A.win + f * A.c.N3 + idx);
        if (A.accumulate)
#pragma unroll
            for (int d = 0; d < 3; d++) prefetch_l2(A.kacc + d * A.c.N3 + idx);
    }

    template <class V>
    __device__ static void site(const Args &A, const V &v, int i, int j, int k, long long idx, Carry &cy,
                                bool first_plane) {
        const FabConsts &c = A.c;
        const long long N3 = c.N3;
        // the momenta and the accumulated currents are loaded first, so their
        // latency passes under the stencil instead of stalling the kicks
        double wv[12], kin[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int f = 0; f < 12; f++) wv[f] = A.win[f * N3 + idx];
        if (A.accumulate) {
#pragma unroll
            for (int d = 0; d < 3; d++) kin[d] = A.kacc[d * N3 + idx];
        }
        double own[12];
#pragma unroll
        for (int f = 0; f < 12; f++) own[f] = v(f);
        if (first_plane) {
            sincos_any(A.qf * v.at(TH, -1, 0, 0), &cy.sm, &cy.cm);
            if (SECOND) sincos_any(A.qx * v.at(TH, -1, 0, 0), &cy.smx, &cy.cmx);
        }
        const double zero[3] = {0.0, 0.0, 0.0};
        double kc[3];
        if (SECOND) {   // the current of the lock partner, same fields, charge qx
            auto lx = [&](int d, double cP[3], double sP[3], double cM[3], double sM[3], double &cW, double &sW) {
                sincos_any(A.qx * v(TH + d), &sW, &cW);
                double cm, sm;
                if (d == 0) { cm = cy.cmx; sm = cy.smx; cy.cmx = cW; cy.smx = sW; }
                else sincos_any(A.qx * nb(v, TH + d, d, -1), &sm, &cm);
#pragma unroll
                for (int a = 0; a < 3; a++) { cP[a] = cW; sP[a] = sW; cM[a] = cm; sM[a] = sm; }
            };
            MultipletOut ox;
            covariant_multiplet<false>(v, 0, own, lx, zero, c.idx1, c.inva, c.eta, ox);
#pragma unroll
            for (int d = 0; d < 3; d++) kc[d] = A.gqx * ox.jlat[d];
        }
        auto links = [&](int d, double cP[3], double sP[3], double cM[3], double sM[3], double &cW, double &sW) {
            sincos_any(A.qf * v(TH + d), &sW, &cW);
            double cm, sm;
            if (d == 0) { cm = cy.cm; sm = cy.sm; cy.cm = cW; cy.sm = sW; }
            else sincos_any(A.qf * nb(v, TH + d, d, -1), &sm, &cm);
#pragma unroll
            for (int a = 0; a < 3; a++) { cP[a] = cW; sP[a] = sW; cM[a] = cm; sM[a] = sm; }
        };
        MultipletOut o;
        covariant_multiplet<false>(v, 0, own, links, zero, c.idx1, c.inva, c.eta, o);
#pragma unroll
        for (int d = 0; d < 3; d++) kc[d] = SECOND ? kc[d] + A.gqf * o.jlat[d] : A.gqf * o.jlat[d];

        double sa[3];
#pragma unroll
        for (int a = 0; a < 3; a++) sa[a] = own[MU + a] * own[MU + a] + own[MV + a] * own[MV + a];
        const double den = 1.0 + c.kappa * (sa[0] * sa[1] * sa[2]);
        const double Vp = 0.5 * c.mu / (den * den);
        double acc[12];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double others = sa[(a + 1) % 3] * sa[(a + 2) % 3];
            const double u = own[MU + a], w = own[MV + a], tu = own[MTU + a], tw = own[MTV + a];
            acc[MU + a] = (o.lsum[MU + a] - 6.0 * u) * c.idx2 - c.m2 * u - 2.0 * Vp * u * others + c.eta * o.curlT[a];
            acc[MV + a] = (o.lsum[MV + a] - 6.0 * w) * c.idx2 - c.m2 * w - 2.0 * Vp * w * others +
                          c.eta * o.curlT[3 + a];
            acc[MTU + a] = (o.lsum[MTU + a] - 6.0 * tu) * c.idx2 - c.mtheta2 * tu + c.eta * o.curlP[a];
            acc[MTV + a] = (o.lsum[MTV + a] - 6.0 * tw) * c.idx2 - c.mtheta2 * tw + c.eta * o.curlP[3 + a];
        }
#pragma unroll
        for (int d = 0; d < 3; d++) A.kacc[d * N3 + idx] = A.accumulate ? kin[d] + kc[d] : kc[d];
        const Leap leap{c.hdt, c.dt, A.first != 0};
        const double dmp = (A.damp && !A.first) ? sponge_at(i, j, k, c.L, c.dx, c.damp_width, c.damp_rate) : 1.0;
        bool bad = false;
#pragma unroll
        for (int f = 0; f < 12; f++) {
            double vv, wn;
            leap(wv[f], acc[f], dmp, &vv, &wn);
            const double x = own[f] + c.dt * wn;
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

// The shared links: plaquette term plus the accumulated currents kick E
// (damped in the sponge), then the angles drift and wrap.
struct LinkPass {
    static constexpr int NR = 3;
    static constexpr int MIN_CTAS = 2;

    struct Args {
        RingSrc<NR> src;      // th
        int N;
        FabConsts c;
        const double *kacc;
        const double *win;    // E: w_n (E_0 on the first launch)
        double *wout, *xout, *sout;
        int *flag;
        int first, sync, damp;
    };

    struct Carry {
        double pm[2];         // plaquette sines (0,1), (2,0) at x - i
    };

    __device__ static void prefetch(const Args &A, long long idx) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            prefetch_l2(A.win + d * A.c.N3 + idx);
            prefetch_l2(A.kacc + d * A.c.N3 + idx);
        }
    }

    template <class V>
    __device__ static void site(const Args &A, const V &v, int i, int j, int k, long long idx, Carry &cy,
                                bool first_plane) {
        const FabConsts &c = A.c;
        const long long N3 = c.N3;
        // E and the accumulated currents first: their latency passes under the staples
        double wv[3], kin[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            wv[d] = A.win[d * N3 + idx];
            kin[d] = A.kacc[d * N3 + idx];
        }
        if (first_plane) {
            cy.pm[0] = plaquette_sin(v, 0, 0, -1, 0, 0);
            cy.pm[1] = plaquette_sin(v, 0, 2, -1, 0, 0);
        }
        double st[3], pat[2];
        staples(v, 0, cy.pm, st, pat);
        cy.pm[0] = pat[0];
        cy.pm[1] = pat[1];
        const Leap leap{c.hdt, c.dt, A.first != 0};
        const double dmp = (A.damp && !A.first) ? sponge_at(i, j, k, c.L, c.dx, c.damp_width, c.damp_rate) : 1.0;
        bool bad = false;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double K = c.stp * st[d] + kin[d];
            double E, Eh;
            leap(wv[d], K, dmp, &E, &Eh);
            const double th = wrap_angle(v(d) + c.gad * Eh);
            st_cs(A.xout + d * N3 + idx, th);
            A.wout[d * N3 + idx] = Eh;
            if (A.sync) {
                st_cs(A.sout + d * N3 + idx, E);
                bad |= !isfinite(th) || !isfinite(E);
            }
        }
        if (A.sync && bad) atomicOr(A.flag, 1);
    }
};

}  // namespace scp
