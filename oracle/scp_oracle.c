/* scp_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's complex (v66) and gauged (v69) lattice
 * leapfrog stepper, kardianos/scp sfa/sim/scp_sim.c, with the gauged
 * extensions (v71 Higgs condensate and second U(1) gauge, v75 three matter
 * fabrics) and the real 6-field mode with its optional terms, bc_type 0
 * (absorbing sphere) or 2 (periodic).  It is the
 * checker for the CUDA library's parity tests and is never part of the
 * product.  Parity of this restatement is pinned against the reference
 * binary itself (oracle/_ref/scp_sim, built from the reference sources by
 * oracle/Makefile) through the fixtures in tests/golden/.
 *
 * Each routine cites the reference function it restates; the arithmetic is
 * written in the same operation order so that the restatement agrees with
 * the reference to rounding (the reference is built with gcc's default FMA
 * contraction, this file with -ffp-contract=off, so agreement is to a few
 * ulps per step, not bitwise).
 */
#include "scp_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846

/* field slots of the packed state: positions q[0..11] = u0..2 v0..2 tu0..2 tv0..2,
 * velocities p[0..11] in the same order */
enum { U0 = 0, V0 = 3, TU0 = 6, TV0 = 9 };

struct orc_state {
    orc_params P;
    long N3;
    double *q[12], *p[12], *a[12];   /* positions, velocities, accelerations (fabric C) */
    double *th[3], *E[3], *K[3];     /* links, electric field, E-kick */
    double *lc[3], *ls[3], *ps[3];   /* scratch: link cos/sin, plaquette sines */
    int higgs, g2on, mf, real;       /* extensions present; real 6-field mode */
    double *mis[3], *hq[3];          /* real mode scratch: Cosserat mismatch, hardening vector */
    double *th2[3], *E2[3], *K2[3], *ps2[3];   /* second gauge */
    double *H, *HV, *HA;                       /* Higgs field, velocity, acceleration */
    double *fq[2][12], *fp[2][12], *fa[2][12]; /* fabrics Q (0) and L (1) */
    double G_offset;
    int cg_iters;
    double *mem;
};

/* ---------------------------------------------------------------- helpers */

typedef struct { long ip, im, jp, jm, kp, km; } nbr_t;

static inline nbr_t nbrs(int N, long idx) {
    const long NN = (long)N * N;
    int i = (int)(idx / NN), j = (int)((idx / N) % N), k = (int)(idx % N);
    int ip = (i + 1) % N, im = (i - 1 + N) % N, jp = (j + 1) % N, jm = (j - 1 + N) % N;
    int kp = (k + 1) % N, km = (k - 1 + N) % N;
    nbr_t n;
    n.ip = (long)ip * NN + (long)j * N + k;  n.im = (long)im * NN + (long)j * N + k;
    n.jp = (long)i * NN + (long)jp * N + k;  n.jm = (long)i * NN + (long)jm * N + k;
    n.kp = (long)i * NN + (long)j * N + kp;  n.km = (long)i * NN + (long)j * N + km;
    return n;
}

/* curl component a of the 3-vector field F at a site
 * (restates curl_component, scp_sim.c:409-415) */
static inline double curl_a(double *const F[3], int a, const nbr_t *n, double idx1) {
    if (a == 0) return (F[2][n->jp] - F[2][n->jm] - F[1][n->kp] + F[1][n->km]) * idx1;
    if (a == 1) return (F[0][n->kp] - F[0][n->km] - F[2][n->ip] + F[2][n->im]) * idx1;
    return (F[1][n->ip] - F[1][n->im] - F[0][n->jp] + F[0][n->jm]) * idx1;
}

static inline double wrap_angle(double v) {
    return v - 2.0 * ORC_PI * rint(v / (2.0 * ORC_PI));
}

/* ---------------------------------------------------------------- forces */

/* compute_forces_complex, scp_sim.c:931-994 */
static void forces_complex(orc_state *s) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long N3 = s->N3;
    const double idx2 = 1.0 / (P->dx * P->dx), idx1 = 1.0 / (2.0 * P->dx);
    const double MU = P->mu, KAPPA = P->kappa, MASS2 = P->m2, MTHETA2 = P->mtheta2, ETA = P->eta;
    double *const *q = s->q;
    double *const *acc = s->a;
    double *const U[3] = {q[0], q[1], q[2]}, *const Vv[3] = {q[3], q[4], q[5]};
    double *const TU[3] = {q[6], q[7], q[8]}, *const TV[3] = {q[9], q[10], q[11]};
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        double u0 = U[0][idx], u1 = U[1][idx], u2 = U[2][idx];
        double v0 = Vv[0][idx], v1 = Vv[1][idx], v2 = Vv[2][idx];
        double s0 = u0 * u0 + v0 * v0, s1 = u1 * u1 + v1 * v1, s2 = u2 * u2 + v2 * v2;
        double sp = s0 * s1 * s2;
        double den = 1.0 + KAPPA * sp;
        double Vp = 0.5 * MU / (den * den);
        double rest[3] = {s1 * s2, s0 * s2, s0 * s1};
        for (int a = 0; a < 3; a++) {
            double x = U[a][idx];
            double lap = (U[a][n.ip] + U[a][n.im] + U[a][n.jp] + U[a][n.jm] + U[a][n.kp] + U[a][n.km]
                          - 6.0 * x) * idx2;
            acc[U0 + a][idx] = lap - MASS2 * x - 2.0 * Vp * x * rest[a] + ETA * curl_a(TU, a, &n, idx1);
            x = Vv[a][idx];
            lap = (Vv[a][n.ip] + Vv[a][n.im] + Vv[a][n.jp] + Vv[a][n.jm] + Vv[a][n.kp] + Vv[a][n.km]
                   - 6.0 * x) * idx2;
            acc[V0 + a][idx] = lap - MASS2 * x - 2.0 * Vp * x * rest[a] + ETA * curl_a(TV, a, &n, idx1);
            x = TU[a][idx];
            lap = (TU[a][n.ip] + TU[a][n.im] + TU[a][n.jp] + TU[a][n.jm] + TU[a][n.kp] + TU[a][n.km]
                   - 6.0 * x) * idx2;
            acc[TU0 + a][idx] = lap - MTHETA2 * x + ETA * curl_a(U, a, &n, idx1);
            x = TV[a][idx];
            lap = (TV[a][n.ip] + TV[a][n.im] + TV[a][n.jp] + TV[a][n.jm] + TV[a][n.kp] + TV[a][n.km]
                   - 6.0 * x) * idx2;
            acc[TV0 + a][idx] = lap - MTHETA2 * x + ETA * curl_a(Vv, a, &n, idx1);
        }
    }
}

static void link_trig(orc_state *s) {
    for (int d = 0; d < 3; d++) {
        double *th = s->th[d], *c = s->lc[d], *sn = s->ls[d];
#pragma omp parallel for schedule(static)
        for (long idx = 0; idx < s->N3; idx++) { c[idx] = cos(th[idx]); sn[idx] = sin(th[idx]); }
    }
}

/* plaquette angle in plane (a,b) at site idx with forward neighbours np[] */
static inline double plaq_angle(double *const th[3], int a, int b, long idx, const long np[3]) {
    return th[a][idx] + th[b][np[a]] - th[a][np[b]] - th[b][idx];
}

/* compute_forces_complex_gauge, scp_sim.c:1053-1263, with its v71 terms:
 * Higgs back-reaction and H_acc (HIG), second gauge (G2: matter transported
 * by th + q_a th2, staples and current of th2 into K2) */
static void forces_gauge(orc_state *s) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long N3 = s->N3;
    const double dx = P->dx, idx2 = 1.0 / (dx * dx), idx1 = 1.0 / (2.0 * dx), inva = 1.0 / dx;
    const double MU = P->mu, KAPPA = P->kappa, MASS2 = P->m2, MTHETA2 = P->mtheta2, ETA = P->eta;
    const double GG = P->g, STP = 1.0 / (GG * dx * dx * dx);
    const int HIG = s->higgs, G2 = s->g2on;
    const double HV = P->higgs_v, HLAM = P->higgs_lam, HKAP = P->higgs_kap;
    const double GG2 = P->g2, STP2 = G2 ? 1.0 / (GG2 * dx * dx * dx) : 0.0;
    static const int pa[3] = {0, 1, 2}, pb[3] = {1, 2, 0};
    static const int ci1[3] = {1, 2, 0}, ci2[3] = {2, 0, 1};

    /* pass A: link cos/sin */
    link_trig(s);
    /* pass B: plaquette sines, planes (0,1) (1,2) (2,0) */
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        long np[3] = {n.ip, n.jp, n.kp};
        for (int p = 0; p < 3; p++) s->ps[p][idx] = sin(plaq_angle(s->th, pa[p], pb[p], idx, np));
        if (G2)
            for (int p = 0; p < 3; p++) s->ps2[p][idx] = sin(plaq_angle(s->th2, pa[p], pb[p], idx, np));
    }
    /* pass C: matter accelerations and E-kick */
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        long np[3] = {n.ip, n.jp, n.kp}, nm[3] = {n.im, n.jm, n.km};
        double fu[6], fv[6];
        for (int a = 0; a < 3; a++) {
            fu[a] = s->q[U0 + a][idx];      fv[a] = s->q[V0 + a][idx];
            fu[3 + a] = s->q[TU0 + a][idx]; fv[3 + a] = s->q[TV0 + a][idx];
        }
        double TRp[3][6], TIp[3][6], TRm[3][6], TIm[3][6], tup[3][3], tvp[3][3];
        for (int d = 0; d < 3; d++) {
            for (int a = 0; a < 3; a++) {
                double cP, sP, cM, sM;
                if (G2) {   /* combined link th + q_a th2 of component a */
                    double php = s->th[d][idx] + P->q2[a] * s->th2[d][idx];
                    double phm = s->th[d][nm[d]] + P->q2[a] * s->th2[d][nm[d]];
                    cP = cos(php); sP = sin(php); cM = cos(phm); sM = sin(phm);
                } else {
                    cP = s->lc[d][idx]; sP = s->ls[d][idx];
                    cM = s->lc[d][nm[d]]; sM = s->ls[d][nm[d]];
                }
                double upn = s->q[U0 + a][np[d]], vpn = s->q[V0 + a][np[d]];
                double umn = s->q[U0 + a][nm[d]], vmn = s->q[V0 + a][nm[d]];
                double tpn = s->q[TU0 + a][np[d]], wpn = s->q[TV0 + a][np[d]];
                double tmn = s->q[TU0 + a][nm[d]], wmn = s->q[TV0 + a][nm[d]];
                TRp[d][a] = cP * upn - sP * vpn;       TIp[d][a] = cP * vpn + sP * upn;
                TRm[d][a] = cM * umn + sM * vmn;       TIm[d][a] = cM * vmn - sM * umn;
                TRp[d][3 + a] = cP * tpn - sP * wpn;   TIp[d][3 + a] = cP * wpn + sP * tpn;
                TRm[d][3 + a] = cM * tmn + sM * wmn;   TIm[d][3 + a] = cM * wmn - sM * tmn;
                tup[d][a] = tpn; tvp[d][a] = wpn;
            }
        }
        double s0 = fu[0] * fu[0] + fv[0] * fv[0];
        double s1 = fu[1] * fu[1] + fv[1] * fv[1];
        double s2 = fu[2] * fu[2] + fv[2] * fv[2];
        double sp = s0 * s1 * s2;
        double den = 1.0 + KAPPA * sp;
        double Vp = 0.5 * MU / (den * den);
        double rest[3] = {s1 * s2, s0 * s2, s0 * s1};
        double hh = HIG ? s->H[idx] * s->H[idx] : 0.0;
        double DcU[3][6], DcV[3][6];
        for (int d = 0; d < 3; d++)
            for (int f = 0; f < 6; f++) {
                DcU[d][f] = (TRp[d][f] - TRm[d][f]) * idx1;
                DcV[d][f] = (TIp[d][f] - TIm[d][f]) * idx1;
            }
        for (int a = 0; a < 3; a++) {
            int d1 = ci1[a], d2 = ci2[a];
            double reDxT = DcU[d1][3 + d2] - DcU[d2][3 + d1];
            double imDxT = DcV[d1][3 + d2] - DcV[d2][3 + d1];
            double reDxP = DcU[d1][d2] - DcU[d2][d1];
            double imDxP = DcV[d1][d2] - DcV[d2][d1];
            double lapUP = (TRp[0][a] + TRm[0][a] + TRp[1][a] + TRm[1][a] + TRp[2][a] + TRm[2][a]
                            - 6.0 * fu[a]) * idx2;
            double lapVP = (TIp[0][a] + TIm[0][a] + TIp[1][a] + TIm[1][a] + TIp[2][a] + TIm[2][a]
                            - 6.0 * fv[a]) * idx2;
            double lapUT = (TRp[0][3 + a] + TRm[0][3 + a] + TRp[1][3 + a] + TRm[1][3 + a]
                            + TRp[2][3 + a] + TRm[2][3 + a] - 6.0 * fu[3 + a]) * idx2;
            double lapVT = (TIp[0][3 + a] + TIm[0][3 + a] + TIp[1][3 + a] + TIm[1][3 + a]
                            + TIp[2][3 + a] + TIm[2][3 + a] - 6.0 * fv[3 + a]) * idx2;
            double au = lapUP - MASS2 * fu[a] - 2.0 * Vp * fu[a] * rest[a] + ETA * reDxT;
            double av = lapVP - MASS2 * fv[a] - 2.0 * Vp * fv[a] * rest[a] + ETA * imDxT;
            if (HIG) {   /* - HKAP hh f prod_rest (scp_sim.c:1196-1200) */
                au = au - HKAP * hh * fu[a] * rest[a];
                av = av - HKAP * hh * fv[a] * rest[a];
            }
            s->a[U0 + a][idx] = au;
            s->a[V0 + a][idx] = av;
            s->a[TU0 + a][idx] = lapUT - MTHETA2 * fu[3 + a] + ETA * reDxP;
            s->a[TV0 + a][idx] = lapVT - MTHETA2 * fv[3 + a] + ETA * imDxP;
        }
        if (HIG) {   /* Hddot = lapH - lam H (H^2 - v^2) - kap s H (:1206-1211) */
            double *H = s->H;
            double lapH = (H[n.ip] + H[n.im] + H[n.jp] + H[n.jm] + H[n.kp] + H[n.km] - 6.0 * H[idx]) * idx2;
            double h = H[idx];
            s->HA[idx] = lapH - HLAM * h * (h * h - HV * HV) - HKAP * sp * h;
        }
        double st2[3] = {0, 0, 0};
        if (G2) {
            double *const *q2 = s->ps2;
            st2[0] = (q2[0][idx] - q2[0][nm[1]]) - (q2[2][idx] - q2[2][nm[2]]);
            st2[1] = -(q2[0][idx] - q2[0][nm[0]]) + (q2[1][idx] - q2[1][nm[2]]);
            st2[2] = (q2[2][idx] - q2[2][nm[0]]) - (q2[1][idx] - q2[1][nm[1]]);
        }
        double *const *ps = s->ps;
        double st[3];
        st[0] = (ps[0][idx] - ps[0][nm[1]]) - (ps[2][idx] - ps[2][nm[2]]);
        st[1] = -(ps[0][idx] - ps[0][nm[0]]) + (ps[1][idx] - ps[1][nm[2]]);
        st[2] = (ps[2][idx] - ps[2][nm[0]]) - (ps[1][idx] - ps[1][nm[1]]);
        for (int d = 0; d < 3; d++) {
            double cP = s->lc[d][idx], sP = s->ls[d][idx];
            double Jg = 0.0;
            for (int a = 0; a < 3; a++) {
                Jg += fu[a] * TIp[d][a] - fv[a] * TRp[d][a];
                Jg += fu[3 + a] * TIp[d][3 + a] - fv[3 + a] * TRp[d][3 + a];
            }
            int d1 = ci1[d], d2 = ci2[d];
            double WpR1 = cP * fu[d2] + sP * fv[d2], WpI1 = cP * fv[d2] - sP * fu[d2];
            double WpR2 = cP * fu[d1] + sP * fv[d1], WpI2 = cP * fv[d1] - sP * fu[d1];
            double T12 = (fu[3 + d1] * TIp[d][d2] - fv[3 + d1] * TRp[d][d2])
                       + (tup[d][d1] * WpI1 - tvp[d][d1] * WpR1);
            double T21 = (fu[3 + d2] * TIp[d][d1] - fv[3 + d2] * TRp[d][d1])
                       + (tup[d][d2] * WpI2 - tvp[d][d2] * WpR2);
            double Jlat = inva * Jg - 0.5 * ETA * (T12 - T21);
            s->K[d][idx] = STP * st[d] + GG * Jlat;
            if (G2) {   /* relative current of the second gauge (:1251-1259) */
                double Jg2 = 0.0;
                for (int a = 0; a < 3; a++) {
                    Jg2 += P->q2[a] * (fu[a] * TIp[d][a] - fv[a] * TRp[d][a]);
                    Jg2 += P->q2[a] * (fu[3 + a] * TIp[d][3 + a] - fv[3 + a] * TRp[d][3 + a]);
                }
                s->K2[d][idx] = STP2 * st2[d] + GG2 * inva * Jg2;
            }
        }
    }
}

/* Matter accelerations of one fabric (view X positions, A accelerations; A
 * = NULL stores none) with charge-q_em links, and the current it adds to the
 * E kick: mode 0 sets K = staples + g q_em J, mode 1 adds g q_em J
 * (force_fabric_gauged_accum, scp_sim.c:1274-1382) */
static void fabric_accum(orc_state *s, double *const *X, double *const *A, double q_em, int mode) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long N3 = s->N3;
    const double dx = P->dx, idx2 = 1.0 / (dx * dx), idx1 = 1.0 / (2.0 * dx), inva = 1.0 / dx;
    const double MU = P->mu, KAPPA = P->kappa, MASS2 = P->m2, MTHETA2 = P->mtheta2, ETA = P->eta;
    const double GG = P->g, STP = 1.0 / (GG * dx * dx * dx);
    static const int ci1[3] = {1, 2, 0}, ci2[3] = {2, 0, 1};
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        long np[3] = {n.ip, n.jp, n.kp}, nm[3] = {n.im, n.jm, n.km};
        double fu[6], fv[6];
        for (int a = 0; a < 3; a++) {
            fu[a] = X[U0 + a][idx];      fv[a] = X[V0 + a][idx];
            fu[3 + a] = X[TU0 + a][idx]; fv[3 + a] = X[TV0 + a][idx];
        }
        double TRp[3][6], TIp[3][6], TRm[3][6], TIm[3][6], tup[3][3], tvp[3][3];
        for (int d = 0; d < 3; d++) {
            double cP = cos(q_em * s->th[d][idx]), sP = sin(q_em * s->th[d][idx]);
            double cM = cos(q_em * s->th[d][nm[d]]), sM = sin(q_em * s->th[d][nm[d]]);
            for (int a = 0; a < 3; a++) {
                double upn = X[U0 + a][np[d]], vpn = X[V0 + a][np[d]];
                double umn = X[U0 + a][nm[d]], vmn = X[V0 + a][nm[d]];
                double tpn = X[TU0 + a][np[d]], wpn = X[TV0 + a][np[d]];
                double tmn = X[TU0 + a][nm[d]], wmn = X[TV0 + a][nm[d]];
                TRp[d][a] = cP * upn - sP * vpn;       TIp[d][a] = cP * vpn + sP * upn;
                TRm[d][a] = cM * umn + sM * vmn;       TIm[d][a] = cM * vmn - sM * umn;
                TRp[d][3 + a] = cP * tpn - sP * wpn;   TIp[d][3 + a] = cP * wpn + sP * tpn;
                TRm[d][3 + a] = cM * tmn + sM * wmn;   TIm[d][3 + a] = cM * wmn - sM * tmn;
                tup[d][a] = tpn; tvp[d][a] = wpn;
            }
        }
        double s0 = fu[0] * fu[0] + fv[0] * fv[0];
        double s1 = fu[1] * fu[1] + fv[1] * fv[1];
        double s2 = fu[2] * fu[2] + fv[2] * fv[2];
        double sp = s0 * s1 * s2;
        double den = 1.0 + KAPPA * sp;
        double Vp = 0.5 * MU / (den * den);
        double rest[3] = {s1 * s2, s0 * s2, s0 * s1};
        double DcU[3][6], DcV[3][6];
        for (int d = 0; d < 3; d++)
            for (int f = 0; f < 6; f++) {
                DcU[d][f] = (TRp[d][f] - TRm[d][f]) * idx1;
                DcV[d][f] = (TIp[d][f] - TIm[d][f]) * idx1;
            }
        if (A)
            for (int a = 0; a < 3; a++) {
                int d1 = ci1[a], d2 = ci2[a];
                double reDxT = DcU[d1][3 + d2] - DcU[d2][3 + d1];
                double imDxT = DcV[d1][3 + d2] - DcV[d2][3 + d1];
                double reDxP = DcU[d1][d2] - DcU[d2][d1];
                double imDxP = DcV[d1][d2] - DcV[d2][d1];
                double lapUP = (TRp[0][a] + TRm[0][a] + TRp[1][a] + TRm[1][a] + TRp[2][a] + TRm[2][a]
                                - 6.0 * fu[a]) * idx2;
                double lapVP = (TIp[0][a] + TIm[0][a] + TIp[1][a] + TIm[1][a] + TIp[2][a] + TIm[2][a]
                                - 6.0 * fv[a]) * idx2;
                double lapUT = (TRp[0][3 + a] + TRm[0][3 + a] + TRp[1][3 + a] + TRm[1][3 + a]
                                + TRp[2][3 + a] + TRm[2][3 + a] - 6.0 * fu[3 + a]) * idx2;
                double lapVT = (TIp[0][3 + a] + TIm[0][3 + a] + TIp[1][3 + a] + TIm[1][3 + a]
                                + TIp[2][3 + a] + TIm[2][3 + a] - 6.0 * fv[3 + a]) * idx2;
                A[U0 + a][idx] = lapUP - MASS2 * fu[a] - 2.0 * Vp * fu[a] * rest[a] + ETA * reDxT;
                A[V0 + a][idx] = lapVP - MASS2 * fv[a] - 2.0 * Vp * fv[a] * rest[a] + ETA * imDxT;
                A[TU0 + a][idx] = lapUT - MTHETA2 * fu[3 + a] + ETA * reDxP;
                A[TV0 + a][idx] = lapVT - MTHETA2 * fv[3 + a] + ETA * imDxP;
            }
        double *const *ps = s->ps;
        double st[3];
        st[0] = (ps[0][idx] - ps[0][nm[1]]) - (ps[2][idx] - ps[2][nm[2]]);
        st[1] = -(ps[0][idx] - ps[0][nm[0]]) + (ps[1][idx] - ps[1][nm[2]]);
        st[2] = (ps[2][idx] - ps[2][nm[0]]) - (ps[1][idx] - ps[1][nm[1]]);
        for (int d = 0; d < 3; d++) {
            double cP = cos(q_em * s->th[d][idx]), sP = sin(q_em * s->th[d][idx]);
            double Jg = 0.0;
            for (int a = 0; a < 3; a++) {
                Jg += fu[a] * TIp[d][a] - fv[a] * TRp[d][a];
                Jg += fu[3 + a] * TIp[d][3 + a] - fv[3 + a] * TRp[d][3 + a];
            }
            int d1 = ci1[d], d2 = ci2[d];
            double WpR1 = cP * fu[d2] + sP * fv[d2], WpI1 = cP * fv[d2] - sP * fu[d2];
            double WpR2 = cP * fu[d1] + sP * fv[d1], WpI2 = cP * fv[d1] - sP * fu[d1];
            double T12 = (fu[3 + d1] * TIp[d][d2] - fv[3 + d1] * TRp[d][d2])
                       + (tup[d][d1] * WpI1 - tvp[d][d1] * WpR1);
            double T21 = (fu[3 + d2] * TIp[d][d1] - fv[3 + d2] * TRp[d][d1])
                       + (tup[d][d2] * WpI2 - tvp[d][d2] * WpR2);
            double Jlat = inva * Jg - 0.5 * ETA * (T12 - T21);
            double jterm = GG * q_em * Jlat;
            if (mode == 0) s->K[d][idx] = STP * st[d] + jterm;
            else s->K[d][idx] += jterm;
        }
    }
}

/* mf_lock_copy_CQ, scp_sim.c:150-172: Q <- C, fields, velocities, accelerations */
static void lock_copy(orc_state *s) {
    size_t bytes = s->N3 * sizeof(double);
    for (int f = 0; f < 12; f++) {
        memcpy(s->fq[0][f], s->q[f], bytes);
        memcpy(s->fp[0][f], s->p[f], bytes);
        memcpy(s->fa[0][f], s->a[f], bytes);
    }
}

/* compute_forces_complex_gauge_mf, scp_sim.c:1390-1433 */
static void forces_mf(orc_state *s) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long N3 = s->N3;
    static const int pa[3] = {0, 1, 2}, pb[3] = {1, 2, 0};
    link_trig(s);
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        long np[3] = {n.ip, n.jp, n.kp};
        for (int p = 0; p < 3; p++) s->ps[p][idx] = sin(plaq_angle(s->th, pa[p], pb[p], idx, np));
    }
    fabric_accum(s, s->q, s->a, P->q_fab[0], 0);
    if (P->mf_lock) fabric_accum(s, s->q, s->a, P->q_fab[1], 1);
    else fabric_accum(s, s->fq[0], s->fa[0], P->q_fab[1], 1);
    fabric_accum(s, s->fq[1], s->fa[1], P->q_fab[2], 1);
    if (P->mf_lock) lock_copy(s);
}

/* compute_forces, scp_sim.c:743-929: the real 6-field mode (phi = u, theta =
 * tu; v = tv = 0), its mass modes 1 and 3, chiral helicity kappa_h, Cosserat
 * strain alpha_cs and curl-squared hardening beta_h (two passes over the
 * mismatch M and hardening vector Q) */
static void forces_real(orc_state *s) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long N3 = s->N3;
    const double idx2 = 1.0 / (P->dx * P->dx), idx1 = 1.0 / (2.0 * P->dx);
    const double MU = P->mu, KAPPA = P->kappa, MASS2 = P->m2, MTHETA2 = P->mtheta2, ETA = P->eta;
    const double KH = P->kappa_h, ACS = P->alpha_cs, BH = P->beta_h;
    const int MODE = P->mode;
    const double KG = P->kappa_gamma, IA = P->inv_alpha, IB = P->inv_beta;
    double *const *phi = s->q + U0, *const *th = s->q + TU0;
    if (ACS != 0 || BH != 0) {
#pragma omp parallel for schedule(static)
        for (long idx = 0; idx < N3; idx++) {
            nbr_t n = nbrs(N, idx);
            double cp0 = curl_a(phi, 0, &n, idx1), cp1 = curl_a(phi, 1, &n, idx1), cp2 = curl_a(phi, 2, &n, idx1);
            if (ACS != 0) {
                s->mis[0][idx] = cp0 * 0.5 - th[0][idx];
                s->mis[1][idx] = cp1 * 0.5 - th[1][idx];
                s->mis[2][idx] = cp2 * 0.5 - th[2][idx];
            }
            if (BH != 0) {
                double t0 = th[0][idx], t1 = th[1][idx], t2 = th[2][idx];
                double T2 = t0 * t0 + t1 * t1 + t2 * t2;
                double coeff = 0.5 * BH * T2;
                s->hq[0][idx] = coeff * cp0;
                s->hq[1][idx] = coeff * cp1;
                s->hq[2][idx] = coeff * cp2;
            }
        }
    }
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        double p0 = phi[0][idx], p1 = phi[1][idx], p2 = phi[2][idx];
        double sig = p0 * p0 + p1 * p1 + p2 * p2;
        double me2 = (MODE == 1) ? IA / (1.0 + IB * sig) : MASS2;
        double keff = (MODE == 3) ? KAPPA / (1.0 + KG * sig) : KAPPA;
        double Pp = p0 * p1 * p2, P2 = Pp * Pp;
        double den = 1.0 + keff * P2;
        double dVdP = MU * Pp / (den * den);
        double t2c = 0;
        if (MODE == 3 && KG > 0) {
            double D = 1.0 + KG * sig + KAPPA * P2;
            t2c = MU * KG * KAPPA * P2 * P2 / (D * D);
        }
        double curl_phi[3] = {curl_a(phi, 0, &n, idx1), curl_a(phi, 1, &n, idx1), curl_a(phi, 2, &n, idx1)};
        double h = p0 * curl_phi[0] + p1 * curl_phi[1] + p2 * curl_phi[2];
        double dP2dx = 0, dP2dy = 0, dP2dz = 0;
        if (KH != 0) {
            double Pip = phi[0][n.ip] * phi[1][n.ip] * phi[2][n.ip], Pim = phi[0][n.im] * phi[1][n.im] * phi[2][n.im];
            double Pjp = phi[0][n.jp] * phi[1][n.jp] * phi[2][n.jp], Pjm = phi[0][n.jm] * phi[1][n.jm] * phi[2][n.jm];
            double Pkp = phi[0][n.kp] * phi[1][n.kp] * phi[2][n.kp], Pkm = phi[0][n.km] * phi[1][n.km] * phi[2][n.km];
            dP2dx = (Pip * Pip - Pim * Pim) * idx1;
            dP2dy = (Pjp * Pjp - Pjm * Pjm) * idx1;
            dP2dz = (Pkp * Pkp - Pkm * Pkm) * idx1;
        }
        double curl_M[3] = {0, 0, 0}, curl_Q[3] = {0, 0, 0};
        if (ACS != 0)
            for (int a = 0; a < 3; a++) curl_M[a] = curl_a(s->mis, a, &n, idx1);
        if (BH != 0)
            for (int a = 0; a < 3; a++) curl_Q[a] = curl_a(s->hq, a, &n, idx1);
        double curl_sq = curl_phi[0] * curl_phi[0] + curl_phi[1] * curl_phi[1] + curl_phi[2] * curl_phi[2];
        for (int a = 0; a < 3; a++) {
            double lap = (phi[a][n.ip] + phi[a][n.im] + phi[a][n.jp] + phi[a][n.jm] + phi[a][n.kp] + phi[a][n.km]
                          - 6.0 * phi[a][idx]) * idx2;
            double dPda = (a == 0) ? p1 * p2 : (a == 1) ? p0 * p2 : p0 * p1;
            double ct = curl_a(th, a, &n, idx1);
            double chiral = 0;
            if (KH != 0) {
                double t1 = 2.0 * Pp * dPda * h, t2 = 2.0 * P2 * curl_phi[a], t3;
                if (a == 0) t3 = -(dP2dz * p1 - dP2dy * p2);
                else if (a == 1) t3 = -(dP2dx * p2 - dP2dz * p0);
                else t3 = -(dP2dy * p0 - dP2dx * p1);
                chiral = KH * (t1 + t2 + t3);
            }
            double cosserat_phi = -ACS * curl_M[a];
            double harden_phi = -2.0 * curl_Q[a];
            s->a[U0 + a][idx] = lap - me2 * phi[a][idx] - dVdP * dPda - t2c * phi[a][idx] + ETA * ct + chiral
                              + cosserat_phi + harden_phi;
        }
        for (int a = 0; a < 3; a++) {
            double lapt = (th[a][n.ip] + th[a][n.im] + th[a][n.jp] + th[a][n.jm] + th[a][n.kp] + th[a][n.km]
                           - 6.0 * th[a][idx]) * idx2;
            double cp = curl_a(phi, a, &n, idx1);
            double cosserat_theta = (ACS != 0) ? 2.0 * ACS * s->mis[a][idx] : 0.0;
            double harden_theta = -BH * curl_sq * th[a][idx];
            s->a[TU0 + a][idx] = lapt - MTHETA2 * th[a][idx] + ETA * cp + cosserat_theta + harden_theta;
        }
    }
}

static void forces(orc_state *s) {
    if (s->real) forces_real(s);
    else if (s->mf) forces_mf(s);
    else if (s->P.gauge) forces_gauge(s);
    else forces_complex(s);
}

/* ---------------------------------------------------------------- stepping */

/* apply_damping, scp_sim.c:1440-1473 (complex + gauged members only) */
static void damping(orc_state *s) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long NN = (long)N * N;
    const double L = P->L, dx = P->dx, DW = P->damp_width, DR = P->damp_rate;
    if (DW <= 0 || DR <= 0) return;
    const double R_damp = L - DW;
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < s->N3; idx++) {
        int i = (int)(idx / NN), j = (int)((idx / N) % N), k = (int)(idx % N);
        double x = -L + i * dx, y = -L + j * dx, z = -L + k * dx;
        double r = sqrt(x * x + y * y + z * z);
        if (r > R_damp) {
            double sc = (r - R_damp) / DW;
            if (sc > 1) sc = 1;
            double d = 1.0 - DR * sc * sc;
            for (int f = 0; f < 12; f++) s->p[f][idx] *= d;
            if (P->gauge) for (int c = 0; c < 3; c++) s->E[c][idx] *= d;
            if (s->mf)   /* Q and L velocities too (not E2, not the Higgs) */
                for (int fb = 0; fb < 2; fb++)
                    for (int f = 0; f < 12; f++) s->fp[fb][f][idx] *= d;
        }
    }
}

static void axpy(double *v, const double *a, double h, long n) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) v[i] += h * a[i];
}

/* stage 1 / stage 4 kicks of verlet_step (scp_sim.c:1590-1620, :1670-1705):
 * matter of C (and Q unless locked, and L), E, E2, Hdot; with three fabrics
 * and the lock, stage 4 copies C into Q before the E kick */
static void half_kick(orc_state *s, double hdt, int stage4) {
    for (int f = 0; f < 12; f++) axpy(s->p[f], s->a[f], hdt, s->N3);
    if (s->mf) {
        if (!s->P.mf_lock)
            for (int f = 0; f < 12; f++) axpy(s->fp[0][f], s->fa[0][f], hdt, s->N3);
        for (int f = 0; f < 12; f++) axpy(s->fp[1][f], s->fa[1][f], hdt, s->N3);
        if (stage4 && s->P.mf_lock) lock_copy(s);
    }
    if (s->P.gauge)
        for (int c = 0; c < 3; c++) axpy(s->E[c], s->K[c], hdt, s->N3);
    if (s->g2on)
        for (int c = 0; c < 3; c++) axpy(s->E2[c], s->K2[c], hdt, s->N3);
    if (s->higgs) axpy(s->HV, s->HA, hdt, s->N3);
}

/* verlet_step, scp_sim.c:1583-1716: kick, drift (+ link drift and wrap),
 * forces, kick, boundary */
static void verlet(orc_state *s) {
    const double dt = s->P.dt, hdt = 0.5 * dt;
    half_kick(s, hdt, 0);
    for (int f = 0; f < 12; f++) axpy(s->q[f], s->p[f], dt, s->N3);
    if (s->mf) {
        if (!s->P.mf_lock)
            for (int f = 0; f < 12; f++) axpy(s->fq[0][f], s->fp[0][f], dt, s->N3);
        for (int f = 0; f < 12; f++) axpy(s->fq[1][f], s->fp[1][f], dt, s->N3);
    }
    if (s->P.gauge) {
        const double gad = -s->P.g * s->P.dx * dt;
        for (int c = 0; c < 3; c++) {
            double *th = s->th[c], *E = s->E[c];
#pragma omp parallel for schedule(static)
            for (long i = 0; i < s->N3; i++) th[i] = wrap_angle(th[i] + gad * E[i]);
        }
    }
    if (s->g2on) {
        const double gad2 = -s->P.g2 * s->P.dx * dt;
        for (int c = 0; c < 3; c++) {
            double *th = s->th2[c], *E = s->E2[c];
#pragma omp parallel for schedule(static)
            for (long i = 0; i < s->N3; i++) th[i] = wrap_angle(th[i] + gad2 * E[i]);
        }
    }
    if (s->higgs) axpy(s->H, s->HV, dt, s->N3);
    forces(s);
    half_kick(s, hdt, 1);
    if (s->P.bc_type == 0) damping(s);
}

void orc_step(orc_state *s, int nsteps) {
    for (int n = 0; n < nsteps; n++) verlet(s);
}

/* ---------------------------------------------------------------- Gauss law */

static inline double rho_at(const orc_state *s, long idx) {
    double r = 0;
    for (int a = 0; a < 3; a++)
        r += s->q[U0 + a][idx] * s->p[V0 + a][idx] - s->q[V0 + a][idx] * s->p[U0 + a][idx]
           + s->q[TU0 + a][idx] * s->p[TV0 + a][idx] - s->q[TV0 + a][idx] * s->p[TU0 + a][idx];
    return r;
}

/* Noether density of fabric f (0 = Q, 1 = L) (fabric_rho_at, scp_sim.c:174-180) */
static inline double fabric_rho(const orc_state *s, int f, long idx) {
    double r = 0;
    for (int a = 0; a < 3; a++)
        r += s->fq[f][U0 + a][idx] * s->fp[f][V0 + a][idx] - s->fq[f][V0 + a][idx] * s->fp[f][U0 + a][idx]
           + s->fq[f][TU0 + a][idx] * s->fp[f][TV0 + a][idx] - s->fq[f][TV0 + a][idx] * s->fp[f][TU0 + a][idx];
    return r;
}

/* EM charge density: rho of fabric C, or sum_f q_f rho_f with three fabrics
 * (em_rho_at, scp_sim.c:184-197) */
static inline double em_rho_at(const orc_state *s, long idx) {
    if (!s->mf) return rho_at(s, idx);
    return s->P.q_fab[0] * rho_at(s, idx) + s->P.q_fab[1] * fabric_rho(s, 0, idx) + s->P.q_fab[2] * fabric_rho(s, 1, idx);
}

/* gauss_residual_at, scp_sim.c:2176-2181 */
static inline double gauss_at(const orc_state *s, long idx, const nbr_t *n) {
    double divE = (s->E[0][idx] - s->E[0][n->im] + s->E[1][idx] - s->E[1][n->jm]
                   + s->E[2][idx] - s->E[2][n->km]) / s->P.dx;
    return divE - s->P.g * em_rho_at(s, idx);
}

/* net_charge_check, scp_sim.c:2264-2279: 0 when neutral */
static int net_charge_ok(const orc_state *s) {
    const double dV = s->P.dx * s->P.dx * s->P.dx;
    double qn = 0, qa = 0;
#pragma omp parallel for reduction(+ : qn, qa) schedule(static)
    for (long idx = 0; idx < s->N3; idx++) {
        double r = em_rho_at(s, idx);
        qn += r * dV;
        qa += fabs(r) * dV;
    }
    return !(fabs(qn) > 1e-6 * fmax(qa, 1.0));
}

/* The CG of init_gauss_project (scp_sim.c:2314-2366), also used by
 * init_gauss2_project (:2430-2447): b -= mean(b); solve -lap chi = b on the
 * periodic 7-point Laplacian to 1e-13 max(1, max|b|), chi kept zero-mean.
 * Returns 0 with chi in xv, or -3 when 20000 iterations do not converge. */
static int cg_poisson(const orc_state *s, double *b, double *xv, int *iters) {
    const int N = s->P.N;
    const long N3 = s->N3;
    const double dx = s->P.dx, idx2 = 1.0 / (dx * dx);
    double *r = malloc(N3 * sizeof(double)), *pp = malloc(N3 * sizeof(double));
    double *Ap = malloc(N3 * sizeof(double));
    if (!r || !pp || !Ap) { free(r); free(pp); free(Ap); return -4; }
    double gsum = 0, gmax0 = 0;
#pragma omp parallel for reduction(+ : gsum) schedule(static)
    for (long idx = 0; idx < N3; idx++) gsum += b[idx];
    double gbar = gsum / (double)N3;
#pragma omp parallel for reduction(max : gmax0) schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        b[idx] -= gbar;
        double d = fabs(b[idx]);
        if (d > gmax0) gmax0 = d;
    }
    const double tol = 1e-13 * fmax(1.0, gmax0);
    memcpy(r, b, N3 * sizeof(double));
    memcpy(pp, b, N3 * sizeof(double));
    memset(xv, 0, N3 * sizeof(double));
    double rz = 0;
#pragma omp parallel for reduction(+ : rz) schedule(static)
    for (long idx = 0; idx < N3; idx++) rz += r[idx] * r[idx];
    int it = 0;
    double rmax = gmax0;
    while (rmax > tol && it < 20000) {
        double pAp = 0;
#pragma omp parallel for reduction(+ : pAp) schedule(static)
        for (long idx = 0; idx < N3; idx++) {
            nbr_t n = nbrs(N, idx);
            double lap = (pp[n.ip] + pp[n.im] + pp[n.jp] + pp[n.jm] + pp[n.kp] + pp[n.km] - 6.0 * pp[idx]) * idx2;
            Ap[idx] = -lap;
            pAp += pp[idx] * Ap[idx];
        }
        double alpha = rz / pAp, rz2 = 0, xsum = 0, rm = 0;
#pragma omp parallel for reduction(+ : rz2, xsum) reduction(max : rm) schedule(static)
        for (long idx = 0; idx < N3; idx++) {
            xv[idx] += alpha * pp[idx];
            r[idx] -= alpha * Ap[idx];
            rz2 += r[idx] * r[idx];
            xsum += xv[idx];
            double d = fabs(r[idx]);
            if (d > rm) rm = d;
        }
        double xbar = xsum / (double)N3, beta = rz2 / rz;
#pragma omp parallel for schedule(static)
        for (long idx = 0; idx < N3; idx++) {
            xv[idx] -= xbar;
            pp[idx] = r[idx] + beta * pp[idx];
        }
        rz = rz2;
        rmax = rm;
        it++;
    }
    *iters = it;
    free(r); free(pp); free(Ap);
    return (rmax > tol) ? -3 : 0;
}

/* init_gauss_project, scp_sim.c:2284-2400: CG on -lap chi = G - mean(G),
 * E += forward gradient of chi, freeze G_offset = mean(G) */
static int gauss_project(orc_state *s) {
    const int N = s->P.N;
    const long N3 = s->N3;
    const double dx = s->P.dx;
    double *b = malloc(N3 * sizeof(double)), *xv = malloc(N3 * sizeof(double));
    if (!b || !xv) { free(b); free(xv); return -4; }
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        b[idx] = gauss_at(s, idx, &n);
    }
    int rc = cg_poisson(s, b, xv, &s->cg_iters);
    if (rc == 0) {
#pragma omp parallel for schedule(static)
        for (long idx = 0; idx < N3; idx++) {
            nbr_t n = nbrs(N, idx);
            s->E[0][idx] += (xv[n.ip] - xv[idx]) / dx;
            s->E[1][idx] += (xv[n.jp] - xv[idx]) / dx;
            s->E[2][idx] += (xv[n.kp] - xv[idx]) / dx;
        }
        double osum = 0;
#pragma omp parallel for reduction(+ : osum) schedule(static)
        for (long idx = 0; idx < N3; idx++) {
            nbr_t n = nbrs(N, idx);
            osum += gauss_at(s, idx, &n);
        }
        s->G_offset = osum / (double)N3;
    }
    free(b); free(xv);
    return rc;
}

/* gauss2_residual_at, scp_sim.c:2402-2412: div E2 - g2 sum_a q_a rho_a */
static inline double gauss2_at(const orc_state *s, long idx, const nbr_t *n) {
    double divE = (s->E2[0][idx] - s->E2[0][n->im] + s->E2[1][idx] - s->E2[1][n->jm]
                   + s->E2[2][idx] - s->E2[2][n->km]) / s->P.dx;
    double rho = 0;
    for (int a = 0; a < 3; a++)
        rho += s->P.q2[a] * (s->q[U0 + a][idx] * s->p[V0 + a][idx] - s->q[V0 + a][idx] * s->p[U0 + a][idx]
                             + s->q[TU0 + a][idx] * s->p[TV0 + a][idx] - s->q[TV0 + a][idx] * s->p[TU0 + a][idx]);
    return divE - s->P.g2 * rho;
}

/* init_gauss2_project, scp_sim.c:2414-2458: the same solve, correction into E2 */
static int gauss2_project(orc_state *s) {
    const int N = s->P.N;
    const long N3 = s->N3;
    const double dx = s->P.dx;
    double *b = malloc(N3 * sizeof(double)), *xv = malloc(N3 * sizeof(double));
    if (!b || !xv) { free(b); free(xv); return -4; }
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        b[idx] = gauss2_at(s, idx, &n);
    }
    int it = 0, rc = cg_poisson(s, b, xv, &it);
    if (rc == 0)
#pragma omp parallel for schedule(static)
        for (long idx = 0; idx < N3; idx++) {
            nbr_t n = nbrs(N, idx);
            s->E2[0][idx] += (xv[n.ip] - xv[idx]) / dx;
            s->E2[1][idx] += (xv[n.jp] - xv[idx]) / dx;
            s->E2[2][idx] += (xv[n.kp] - xv[idx]) / dx;
        }
    free(b); free(xv);
    return rc;
}

/* ---------------------------------------------------------------- diagnostics */

/* compute_energy_complex (scp_sim.c:1823-1880) or compute_energy_complex_gauge
 * (:1886-2036) into out[0..10]; theta_rms_complex/P_integrated_complex
 * (:2041-2061) into out[11..12] */
static void diag_energy(orc_state *s, double *out) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long N3 = s->N3;
    const double dx = P->dx, dV = dx * dx * dx, idx1 = 1.0 / (2.0 * dx);
    const double MU = P->mu, KAPPA = P->kappa, MASS2 = P->m2, MTHETA2 = P->mtheta2, ETA = P->eta;
    const int G = P->gauge;
    const double GG = P->g, BPRE = G ? 1.0 / (GG * GG * dx * dx * dx * dx) : 0.0;
    static const int ci1[3] = {1, 2, 0}, ci2[3] = {2, 0, 1};
    double *const U[3] = {s->q[0], s->q[1], s->q[2]}, *const Vv[3] = {s->q[3], s->q[4], s->q[5]};
    double *const TU[3] = {s->q[6], s->q[7], s->q[8]}, *const TV[3] = {s->q[9], s->q[10], s->q[11]};
    if (G) link_trig(s);
    double epk = 0, etk = 0, eg = 0, em = 0, ep = 0, etg = 0, etm = 0, ec = 0, pm = 0, Pm = 0, eem = 0;
#pragma omp parallel for reduction(+ : epk, etk, eg, em, ep, etg, etm, ec, eem) reduction(max : pm, Pm) schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        double s2[3];
        if (!G) {
            for (int a = 0; a < 3; a++) {
                double u = U[a][idx], v = Vv[a][idx], tu = TU[a][idx], tv = TV[a][idx];
                s2[a] = u * u + v * v;
                epk += 0.5 * (s->p[U0 + a][idx] * s->p[U0 + a][idx] + s->p[V0 + a][idx] * s->p[V0 + a][idx]) * dV;
                etk += 0.5 * (s->p[TU0 + a][idx] * s->p[TU0 + a][idx] + s->p[TV0 + a][idx] * s->p[TV0 + a][idx]) * dV;
                double gx = (U[a][n.ip] - U[a][n.im]) * idx1, gy = (U[a][n.jp] - U[a][n.jm]) * idx1;
                double gz = (U[a][n.kp] - U[a][n.km]) * idx1;
                double hx = (Vv[a][n.ip] - Vv[a][n.im]) * idx1, hy = (Vv[a][n.jp] - Vv[a][n.jm]) * idx1;
                double hz = (Vv[a][n.kp] - Vv[a][n.km]) * idx1;
                eg += 0.5 * (gx * gx + gy * gy + gz * gz + hx * hx + hy * hy + hz * hz) * dV;
                em += 0.5 * MASS2 * (u * u + v * v) * dV;
                double tgx = (TU[a][n.ip] - TU[a][n.im]) * idx1, tgy = (TU[a][n.jp] - TU[a][n.jm]) * idx1;
                double tgz = (TU[a][n.kp] - TU[a][n.km]) * idx1;
                double thx = (TV[a][n.ip] - TV[a][n.im]) * idx1, thy = (TV[a][n.jp] - TV[a][n.jm]) * idx1;
                double thz = (TV[a][n.kp] - TV[a][n.km]) * idx1;
                etg += 0.5 * (tgx * tgx + tgy * tgy + tgz * tgz + thx * thx + thy * thy + thz * thz) * dV;
                etm += 0.5 * MTHETA2 * (tu * tu + tv * tv) * dV;
                double mod = sqrt(s2[a]);
                if (mod > pm) pm = mod;
                double ctu = curl_a(TU, a, &n, idx1), ctv = curl_a(TV, a, &n, idx1);
                ec -= ETA * (u * ctu + v * ctv) * dV;
            }
        } else {
            long np[3] = {n.ip, n.jp, n.kp}, nm[3] = {n.im, n.jm, n.km};
            double fu[6], fv[6];
            for (int a = 0; a < 3; a++) {
                fu[a] = U[a][idx]; fv[a] = Vv[a][idx]; fu[3 + a] = TU[a][idx]; fv[3 + a] = TV[a][idx];
            }
            double DcU[3][6], DcV[3][6];
            for (int d = 0; d < 3; d++) {
                double cP = s->lc[d][idx], sP = s->ls[d][idx];
                double cM = s->lc[d][nm[d]], sM = s->ls[d][nm[d]];
                for (int a = 0; a < 3; a++) {
                    double upn = U[a][np[d]], vpn = Vv[a][np[d]], umn = U[a][nm[d]], vmn = Vv[a][nm[d]];
                    double tpn = TU[a][np[d]], wpn = TV[a][np[d]], tmn = TU[a][nm[d]], wmn = TV[a][nm[d]];
                    DcU[d][a] = ((cP * upn - sP * vpn) - (cM * umn + sM * vmn)) * idx1;
                    DcV[d][a] = ((cP * vpn + sP * upn) - (cM * vmn - sM * umn)) * idx1;
                    DcU[d][3 + a] = ((cP * tpn - sP * wpn) - (cM * tmn + sM * wmn)) * idx1;
                    DcV[d][3 + a] = ((cP * wpn + sP * tpn) - (cM * wmn - sM * tmn)) * idx1;
                }
            }
            for (int a = 0; a < 3; a++) {
                s2[a] = fu[a] * fu[a] + fv[a] * fv[a];
                epk += 0.5 * (s->p[U0 + a][idx] * s->p[U0 + a][idx] + s->p[V0 + a][idx] * s->p[V0 + a][idx]) * dV;
                etk += 0.5 * (s->p[TU0 + a][idx] * s->p[TU0 + a][idx] + s->p[TV0 + a][idx] * s->p[TV0 + a][idx]) * dV;
                eg += 0.5 * (DcU[0][a] * DcU[0][a] + DcU[1][a] * DcU[1][a] + DcU[2][a] * DcU[2][a]
                             + DcV[0][a] * DcV[0][a] + DcV[1][a] * DcV[1][a] + DcV[2][a] * DcV[2][a]) * dV;
                em += 0.5 * MASS2 * s2[a] * dV;
                etg += 0.5 * (DcU[0][3 + a] * DcU[0][3 + a] + DcU[1][3 + a] * DcU[1][3 + a]
                              + DcU[2][3 + a] * DcU[2][3 + a] + DcV[0][3 + a] * DcV[0][3 + a]
                              + DcV[1][3 + a] * DcV[1][3 + a] + DcV[2][3 + a] * DcV[2][3 + a]) * dV;
                etm += 0.5 * MTHETA2 * (fu[3 + a] * fu[3 + a] + fv[3 + a] * fv[3 + a]) * dV;
                double mod = sqrt(s2[a]);
                if (mod > pm) pm = mod;
                double reDxT = DcU[ci1[a]][3 + ci2[a]] - DcU[ci2[a]][3 + ci1[a]];
                double imDxT = DcV[ci1[a]][3 + ci2[a]] - DcV[ci2[a]][3 + ci1[a]];
                ec -= ETA * (fu[a] * reDxT + fv[a] * imDxT) * dV;
            }
            double ee = 0.5 * (s->E[0][idx] * s->E[0][idx] + s->E[1][idx] * s->E[1][idx]
                               + s->E[2][idx] * s->E[2][idx]);
            double bb = 0.0;
            static const int pa[3] = {0, 1, 2}, pb[3] = {1, 2, 0};
            for (int p = 0; p < 3; p++) bb += 1.0 - cos(plaq_angle(s->th, pa[p], pb[p], idx, np));
            eem += (ee + BPRE * bb) * dV;
        }
        double sp = s2[0] * s2[1] * s2[2];
        ep += (MU / 2.0) * sp / (1.0 + KAPPA * sp) * dV;
        double Pmod = sqrt(sp);
        if (Pmod > Pm) Pm = Pmod;
    }
    /* v71 Higgs energy density (scp_sim.c:1970-1975): 1/2 Hdot^2 + 1/2 |grad H|^2
     * + (lam/4)(H^2 - v^2)^2 + (kap/2) s H^2; joins E_total only */
    double ehg = 0;
    if (s->higgs) {
        const double HV = P->higgs_v, HLAM = P->higgs_lam, HKAP = P->higgs_kap;
#pragma omp parallel for reduction(+ : ehg) schedule(static)
        for (long idx = 0; idx < N3; idx++) {
            nbr_t n = nbrs(N, idx);
            double sp = 1.0;
            for (int a = 0; a < 3; a++) sp *= U[a][idx] * U[a][idx] + Vv[a][idx] * Vv[a][idx];
            double h = s->H[idx], hv = s->HV[idx];
            double gx = (s->H[n.ip] - s->H[n.im]) * idx1, gy = (s->H[n.jp] - s->H[n.jm]) * idx1;
            double gz = (s->H[n.kp] - s->H[n.km]) * idx1;
            double hd = h * h - HV * HV;
            ehg += (0.5 * hv * hv + 0.5 * (gx * gx + gy * gy + gz * gz) + 0.25 * HLAM * hd * hd
                    + 0.5 * HKAP * sp * h * h) * dV;
        }
    }
    /* v75 fabric L's matter energy with the unit-charge links (:1977-2028) */
    if (s->mf) {
        double *const *X = s->fq[1], *const *Pv = s->fp[1];
        double l_epk = 0, l_eg = 0, l_em = 0, l_ep = 0, l_etk = 0, l_etg = 0, l_etm = 0, l_ec = 0;
#pragma omp parallel for reduction(+ : l_epk, l_eg, l_em, l_ep, l_etk, l_etg, l_etm, l_ec) schedule(static)
        for (long idx = 0; idx < N3; idx++) {
            nbr_t n = nbrs(N, idx);
            long np[3] = {n.ip, n.jp, n.kp}, nm[3] = {n.im, n.jm, n.km};
            double fu[6], fv[6];
            for (int a = 0; a < 3; a++) {
                fu[a] = X[U0 + a][idx]; fv[a] = X[V0 + a][idx];
                fu[3 + a] = X[TU0 + a][idx]; fv[3 + a] = X[TV0 + a][idx];
            }
            double DcU[3][6], DcV[3][6];
            for (int d = 0; d < 3; d++) {
                double cP = s->lc[d][idx], sP = s->ls[d][idx];
                double cM = s->lc[d][nm[d]], sM = s->ls[d][nm[d]];
                for (int a = 0; a < 3; a++) {
                    double upn = X[U0 + a][np[d]], vpn = X[V0 + a][np[d]];
                    double umn = X[U0 + a][nm[d]], vmn = X[V0 + a][nm[d]];
                    double tpn = X[TU0 + a][np[d]], wpn = X[TV0 + a][np[d]];
                    double tmn = X[TU0 + a][nm[d]], wmn = X[TV0 + a][nm[d]];
                    DcU[d][a] = ((cP * upn - sP * vpn) - (cM * umn + sM * vmn)) * idx1;
                    DcV[d][a] = ((cP * vpn + sP * upn) - (cM * vmn - sM * umn)) * idx1;
                    DcU[d][3 + a] = ((cP * tpn - sP * wpn) - (cM * tmn + sM * wmn)) * idx1;
                    DcV[d][3 + a] = ((cP * wpn + sP * tpn) - (cM * wmn - sM * tmn)) * idx1;
                }
            }
            double s2[3];
            for (int a = 0; a < 3; a++) {
                s2[a] = fu[a] * fu[a] + fv[a] * fv[a];
                l_epk += 0.5 * (Pv[U0 + a][idx] * Pv[U0 + a][idx] + Pv[V0 + a][idx] * Pv[V0 + a][idx]) * dV;
                l_etk += 0.5 * (Pv[TU0 + a][idx] * Pv[TU0 + a][idx] + Pv[TV0 + a][idx] * Pv[TV0 + a][idx]) * dV;
                l_eg += 0.5 * (DcU[0][a] * DcU[0][a] + DcU[1][a] * DcU[1][a] + DcU[2][a] * DcU[2][a]
                               + DcV[0][a] * DcV[0][a] + DcV[1][a] * DcV[1][a] + DcV[2][a] * DcV[2][a]) * dV;
                l_em += 0.5 * MASS2 * s2[a] * dV;
                l_etg += 0.5 * (DcU[0][3 + a] * DcU[0][3 + a] + DcU[1][3 + a] * DcU[1][3 + a]
                                + DcU[2][3 + a] * DcU[2][3 + a] + DcV[0][3 + a] * DcV[0][3 + a]
                                + DcV[1][3 + a] * DcV[1][3 + a] + DcV[2][3 + a] * DcV[2][3 + a]) * dV;
                l_etm += 0.5 * MTHETA2 * (fu[3 + a] * fu[3 + a] + fv[3 + a] * fv[3 + a]) * dV;
                double reDxT = DcU[ci1[a]][3 + ci2[a]] - DcU[ci2[a]][3 + ci1[a]];
                double imDxT = DcV[ci1[a]][3 + ci2[a]] - DcV[ci2[a]][3 + ci1[a]];
                l_ec -= ETA * (fu[a] * reDxT + fv[a] * imDxT) * dV;
            }
            double sp = s2[0] * s2[1] * s2[2];
            l_ep += (MU / 2.0) * sp / (1.0 + KAPPA * sp) * dV;
        }
        epk += l_epk; etk += l_etk; eg += l_eg; em += l_em; ep += l_ep;
        etg += l_etg; etm += l_etm; ec += l_ec;
    }
    double trs = 0, pint = 0;
#pragma omp parallel for reduction(+ : trs, pint) schedule(static)
    for (long i = 0; i < N3; i++) {
        for (int a = 0; a < 3; a++) trs += TU[a][i] * TU[a][i] + TV[a][i] * TV[a][i];
        double a0 = U[0][i] * U[0][i] + Vv[0][i] * Vv[0][i];
        double a1 = U[1][i] * U[1][i] + Vv[1][i] * Vv[1][i];
        double a2 = U[2][i] * U[2][i] + Vv[2][i] * Vv[2][i];
        pint += sqrt(a0 * a1 * a2) * dV;
    }
    out[0] = epk; out[1] = etk; out[2] = eg; out[3] = em; out[4] = ep;
    out[5] = etg; out[6] = etm; out[7] = ec;
    out[8] = epk + etk + eg + em + ep + etg + etm + ec + eem + ehg;
    out[9] = pm; out[10] = Pm; out[11] = pint; out[12] = sqrt(trs / (6.0 * N3));
}

/* compute_charges, scp_sim.c:2074-2169, into out[13..23] and out[28..30] */
static void diag_charges(orc_state *s, double *out) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long NN = (long)N * N, N3 = s->N3;
    const double L = P->L, dx = P->dx, dV = dx * dx * dx, R2 = P->qdiag_radius * P->qdiag_radius;
    double qp = 0, qt = 0, smax = 0, M0 = 0, cx = 0, cy = 0, cz = 0, qc = 0, qp0 = 0, qp1 = 0, qp2 = 0;
#pragma omp parallel for reduction(+ : qp, qt, M0, cx, cy, cz, qc, qp0, qp1, qp2) reduction(max : smax) schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        int i = (int)(idx / NN), j = (int)((idx / N) % N), k = (int)(idx % N);
        double x = -L + i * dx, y = -L + j * dx, z = -L + k * dx;
        double rho2 = 0, sp = 1.0, qpv = 0, qtv = 0;
        for (int a = 0; a < 3; a++) {
            double u = s->q[U0 + a][idx], v = s->q[V0 + a][idx];
            double ud = s->p[U0 + a][idx], vd = s->p[V0 + a][idx];
            double tu = s->q[TU0 + a][idx], tv = s->q[TV0 + a][idx];
            double tud = s->p[TU0 + a][idx], tvd = s->p[TV0 + a][idx];
            double qa = u * vd - v * ud;
            qpv += qa;
            if (a == 0) qp0 += qa; else if (a == 1) qp1 += qa; else qp2 += qa;
            qtv += tu * tvd - tv * tud;
            double s2a = u * u + v * v;
            rho2 += s2a;
            sp *= s2a;
        }
        qp += qpv; qt += qtv;
        if (x * x + y * y + z * z <= R2) qc += qpv + qtv;
        if (sp > smax) smax = sp;
        M0 += rho2;
        cx += x * rho2; cy += y * rho2; cz += z * rho2;
    }
    out[13] = qp * dV; out[14] = qt * dV; out[15] = qp * dV + qt * dV; out[16] = smax;
    out[19] = qc * dV;
    out[28] = qp0 * dV; out[29] = qp1 * dV; out[30] = qp2 * dV;
    /* omega_core at the lowest-index voxel with s >= smax*(1-1e-12) */
    long smax_idx = -1;
    const double sthr = smax * (1.0 - 1e-12);
    for (long idx = 0; idx < N3; idx++) {
        double sp = 1.0;
        for (int a = 0; a < 3; a++) {
            double u = s->q[U0 + a][idx], v = s->q[V0 + a][idx];
            sp *= u * u + v * v;
        }
        if (sp >= sthr) { smax_idx = idx; break; }
    }
    out[18] = 0.0;
    if (smax_idx >= 0) {
        double u0 = s->q[U0][smax_idx], v0 = s->q[V0][smax_idx];
        double ud0 = s->p[U0][smax_idx], vd0 = s->p[V0][smax_idx];
        double den = u0 * u0 + v0 * v0;
        if (den >= 1e-20) out[18] = (u0 * vd0 - v0 * ud0) / den;
    }
    int jc = (int)lround(L / dx);
    if (jc < 0) jc = 0; if (jc > N - 1) jc = N - 1;
    int i1 = (int)lround((P->qdiag_probe1 + L) / dx);
    if (i1 < 0) i1 = 0; if (i1 > N - 1) i1 = N - 1;
    int i2 = (int)lround((P->qdiag_probe2 + L) / dx);
    if (i2 < 0) i2 = 0; if (i2 > N - 1) i2 = N - 1;
    long p1 = (long)i1 * NN + (long)jc * N + jc, p2 = (long)i2 * NN + (long)jc * N + jc;
    out[20] = s->q[TU0 + 1][p1]; out[21] = s->q[TV0 + 1][p1];
    out[22] = s->q[TU0 + 1][p2]; out[23] = s->q[TV0 + 1][p2];
    M0 *= dV;
    if (M0 < 1e-30) { out[17] = 0; return; }
    cx = cx * dV / M0; cy = cy * dV / M0; cz = cz * dV / M0;
    double rsum = 0;
#pragma omp parallel for reduction(+ : rsum) schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        int i = (int)(idx / NN), j = (int)((idx / N) % N), k = (int)(idx % N);
        double x = -L + i * dx, y = -L + j * dx, z = -L + k * dx;
        double rho2 = 0;
        for (int a = 0; a < 3; a++) {
            double u = s->q[U0 + a][idx], v = s->q[V0 + a][idx];
            rho2 += u * u + v * v;
        }
        rsum += ((x - cx) * (x - cx) + (y - cy) * (y - cy) + (z - cz) * (z - cz)) * rho2;
    }
    out[17] = sqrt(rsum * dV / M0);
}

/* compute_gauss, scp_sim.c:2186-2243, into out[24..27] */
static void diag_gauss(orc_state *s, double *out) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long NN = (long)N * N, N3 = s->N3;
    const double L = P->L, dx = P->dx, dV = dx * dx * dx, GG = P->g, OFF = s->G_offset;
    const double Rint = (P->bc_type == 0) ? (L - P->damp_width - dx) : 1e300, Rint2 = Rint * Rint;
    const double Rcube = P->qdiag_radius;
    static const int pa[3] = {0, 1, 2}, pb[3] = {1, 2, 0};
    double gmax = 0, gl2 = 0, eem = 0, fsum = 0;
    long nOmega = 0, nC = 0;
#pragma omp parallel for reduction(+ : gl2, eem, fsum, nOmega, nC) reduction(max : gmax) schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        int i = (int)(idx / NN), j = (int)((idx / N) % N), k = (int)(idx % N);
        nbr_t n = nbrs(N, idx);
        long np[3] = {n.ip, n.jp, n.kp};
        double x = -L + i * dx, y = -L + j * dx, z = -L + k * dx;
        double divE = (s->E[0][idx] - s->E[0][n.im] + s->E[1][idx] - s->E[1][n.jm]
                       + s->E[2][idx] - s->E[2][n.km]) / dx;
        double G = gauss_at(s, idx, &n);
        if (x * x + y * y + z * z < Rint2) {
            double d = fabs(G - OFF);
            if (d > gmax) gmax = d;
            gl2 += (G - OFF) * (G - OFF);
            nOmega++;
        }
        double ee = 0.5 * (s->E[0][idx] * s->E[0][idx] + s->E[1][idx] * s->E[1][idx]
                           + s->E[2][idx] * s->E[2][idx]);
        if (GG != 0) {
            double bb = 0;
            for (int p = 0; p < 3; p++) bb += 1.0 - cos(plaq_angle(s->th, pa[p], pb[p], idx, np));
            ee += bb / (GG * GG * dx * dx * dx * dx);
        }
        eem += ee * dV;
        if (fabs(x) <= Rcube && fabs(y) <= Rcube && fabs(z) <= Rcube) { fsum += divE * dV; nC++; }
    }
    out[24] = gmax;
    out[25] = (nOmega > 0) ? sqrt(gl2 / (double)nOmega) : 0.0;
    out[26] = eem;
    out[27] = (GG != 0) ? (fsum - OFF * (double)nC * dV) / GG : 0.0;
}

/* compute_energy, theta_rms and P_integrated of the real mode
 * (scp_sim.c:1722-1816) into out[0..12] */
static void diag_energy_real(orc_state *s, double *out) {
    const orc_params *P = &s->P;
    const int N = P->N;
    const long N3 = s->N3;
    const double dx = P->dx, dV = dx * dx * dx, idx1 = 1.0 / (2.0 * dx);
    const double MU = P->mu, KAPPA = P->kappa, MASS2 = P->m2, MTHETA2 = P->mtheta2, ETA = P->eta;
    const int MODE = P->mode;
    const double KG = P->kappa_gamma;
    double *const *phi = s->q + U0, *const *th = s->q + TU0, *const *pv = s->p + U0, *const *tv = s->p + TU0;
    double epk = 0, etk = 0, eg = 0, em = 0, ep = 0, etg = 0, etm = 0, ec = 0, pm = 0, Pm = 0;
#pragma omp parallel for reduction(+ : epk, etk, eg, em, ep, etg, etm, ec) reduction(max : pm, Pm) schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        double p0 = phi[0][idx], p1 = phi[1][idx], p2 = phi[2][idx];
        double sig = p0 * p0 + p1 * p1 + p2 * p2;
        double me2 = (MODE == 1) ? P->inv_alpha / (1.0 + P->inv_beta * sig) : MASS2;
        double keff = (MODE == 3) ? KAPPA / (1.0 + KG * sig) : KAPPA;
        for (int a = 0; a < 3; a++) {
            epk += 0.5 * pv[a][idx] * pv[a][idx] * dV;
            etk += 0.5 * tv[a][idx] * tv[a][idx] * dV;
            double gx = (phi[a][n.ip] - phi[a][n.im]) * idx1, gy = (phi[a][n.jp] - phi[a][n.jm]) * idx1;
            double gz = (phi[a][n.kp] - phi[a][n.km]) * idx1;
            eg += 0.5 * (gx * gx + gy * gy + gz * gz) * dV;
            em += 0.5 * me2 * phi[a][idx] * phi[a][idx] * dV;
            double tgx = (th[a][n.ip] - th[a][n.im]) * idx1, tgy = (th[a][n.jp] - th[a][n.jm]) * idx1;
            double tgz = (th[a][n.kp] - th[a][n.km]) * idx1;
            etg += 0.5 * (tgx * tgx + tgy * tgy + tgz * tgz) * dV;
            etm += 0.5 * MTHETA2 * th[a][idx] * th[a][idx] * dV;
            double ap = fabs(phi[a][idx]);
            if (ap > pm) pm = ap;
        }
        double Pp = p0 * p1 * p2, P2 = Pp * Pp;
        if (MODE == 3) {
            double D = 1.0 + KG * sig + KAPPA * P2;
            ep += (MU / 2.0) * P2 * (1.0 + KG * sig) / D * dV;
        } else {
            ep += (MU / 2.0) * P2 / (1.0 + keff * P2) * dV;
        }
        double Pa = fabs(Pp);
        if (Pa > Pm) Pm = Pa;
        double cx0 = curl_a(phi, 0, &n, idx1), cx1 = curl_a(phi, 1, &n, idx1), cx2 = curl_a(phi, 2, &n, idx1);
        if (P->alpha_cs != 0) {   /* alpha |curl(phi)/2 - theta|^2 */
            double m0 = cx0 * 0.5 - th[0][idx], m1 = cx1 * 0.5 - th[1][idx], m2c = cx2 * 0.5 - th[2][idx];
            ep += P->alpha_cs * (m0 * m0 + m1 * m1 + m2c * m2c) * dV;
        }
        if (P->beta_h != 0) {     /* (beta/2) |theta|^2 |curl phi|^2 */
            double csq = cx0 * cx0 + cx1 * cx1 + cx2 * cx2;
            double T2 = th[0][idx] * th[0][idx] + th[1][idx] * th[1][idx] + th[2][idx] * th[2][idx];
            ep += 0.5 * P->beta_h * T2 * csq * dV;
        }
        if (P->kappa_h != 0) {    /* kappa_h P^2 phi . curl phi */
            double hel = p0 * cx0 + p1 * cx1 + p2 * cx2;
            ep += P->kappa_h * P2 * hel * dV;
        }
        for (int a = 0; a < 3; a++) ec -= ETA * phi[a][idx] * curl_a(th, a, &n, idx1) * dV;
    }
    double trs = 0, pint = 0;
#pragma omp parallel for reduction(+ : trs, pint) schedule(static)
    for (long i = 0; i < N3; i++) {
        for (int a = 0; a < 3; a++) trs += th[a][i] * th[a][i];
        pint += fabs(phi[0][i] * phi[1][i] * phi[2][i]) * dV;
    }
    out[0] = epk; out[1] = etk; out[2] = eg; out[3] = em; out[4] = ep;
    out[5] = etg; out[6] = etm; out[7] = ec;
    out[8] = epk + etk + eg + em + ep + etg + etm + ec;
    out[9] = pm; out[10] = Pm; out[11] = pint; out[12] = sqrt(trs / (3.0 * N3));
}

/* compute_mf_charges, scp_sim.c:2247-2261, into out[31..34] */
static void diag_mf_charges(orc_state *s, double *out) {
    const double dV = s->P.dx * s->P.dx * s->P.dx;
    double sc = 0, sq = 0, sl = 0, se = 0;
#pragma omp parallel for reduction(+ : sc, sq, sl, se) schedule(static)
    for (long idx = 0; idx < s->N3; idx++) {
        double rc = rho_at(s, idx), rq = fabric_rho(s, 0, idx), rl = fabric_rho(s, 1, idx);
        sc += rc; sq += rq; sl += rl;
        se += s->P.q_fab[0] * rc + s->P.q_fab[1] * rq + s->P.q_fab[2] * rl;
    }
    out[31] = sc * dV; out[32] = sq * dV; out[33] = sl * dV; out[34] = se * dV;
}

int orc_diag(orc_state *s, double *out) {
    if (s->real) {
        for (int i = 0; i < 13; i++) out[i] = 0.0;
        diag_energy_real(s, out);
        return 13;
    }
    const int n = s->mf ? 35 : 31;
    for (int i = 0; i < n; i++) out[i] = 0.0;
    diag_energy(s, out);
    diag_charges(s, out);
    if (s->P.gauge) diag_gauss(s, out);
    if (s->mf) diag_mf_charges(s, out);
    return n;
}

/* ---------------------------------------------------------------- lifecycle */

/* fabric f (0 = Q, 1 = L) from 24 columns in the complex column order */
static void fabric_in(orc_state *s, int f, const double *const *cols) {
    size_t bytes = s->N3 * sizeof(double);
    for (int a = 0; a < 3; a++) {
        memcpy(s->fq[f][U0 + a], cols[0 + a], bytes);  memcpy(s->fq[f][TU0 + a], cols[3 + a], bytes);
        memcpy(s->fp[f][U0 + a], cols[6 + a], bytes);  memcpy(s->fp[f][TU0 + a], cols[9 + a], bytes);
        memcpy(s->fq[f][V0 + a], cols[12 + a], bytes); memcpy(s->fq[f][TV0 + a], cols[15 + a], bytes);
        memcpy(s->fp[f][V0 + a], cols[18 + a], bytes); memcpy(s->fp[f][TV0 + a], cols[21 + a], bytes);
    }
}

orc_state *orc_create(const orc_params *p, const double *const *cols, int project, int *status) {
    *status = 0;
    if (!p || p->N < 3 || p->dx <= 0 || p->dt <= 0 || (p->gauge && p->g == 0.0)) { *status = -1; return NULL; }
    const int higgs = p->gauge && p->higgs_v > 0, g2on = p->gauge && p->g2 != 0, mf = p->gauge && p->n_fabrics == 3;
    const int real = p->real_fields != 0;
    if (mf && (higgs || g2on)) { *status = -1; return NULL; }   /* cfg_validate, scp_config.h:522-534 */
    if (real && p->gauge) { *status = -1; return NULL; }
    orc_state *s = calloc(1, sizeof(orc_state));
    if (!s) { *status = -4; return NULL; }
    s->P = *p;
    s->N3 = (long)p->N * p->N * p->N;
    s->higgs = higgs; s->g2on = g2on; s->mf = mf; s->real = real;
    int nblk = 36 + (p->gauge ? 18 : 0) + (g2on ? 12 : 0) + (higgs ? 3 : 0) + (mf ? 72 : 0) + (real ? 6 : 0);
    s->mem = calloc((size_t)nblk * s->N3, sizeof(double));
    if (!s->mem) { free(s); *status = -4; return NULL; }
    double *m = s->mem;
    for (int f = 0; f < 12; f++) { s->q[f] = m; m += s->N3; }
    for (int f = 0; f < 12; f++) { s->p[f] = m; m += s->N3; }
    for (int f = 0; f < 12; f++) { s->a[f] = m; m += s->N3; }
    if (p->gauge)
        for (int c = 0; c < 3; c++) {
            s->th[c] = m; m += s->N3; s->E[c] = m; m += s->N3; s->K[c] = m; m += s->N3;
            s->lc[c] = m; m += s->N3; s->ls[c] = m; m += s->N3; s->ps[c] = m; m += s->N3;
        }
    if (g2on)   /* th2 and E2 start at zero: the reference's SFA loader leaves them */
        for (int c = 0; c < 3; c++) {
            s->th2[c] = m; m += s->N3; s->E2[c] = m; m += s->N3;
            s->K2[c] = m; m += s->N3; s->ps2[c] = m; m += s->N3;
        }
    if (higgs) { s->H = m; m += s->N3; s->HV = m; m += s->N3; s->HA = m; m += s->N3; }
    if (mf)
        for (int fb = 0; fb < 2; fb++)
            for (int f = 0; f < 12; f++) {
                s->fq[fb][f] = m; m += s->N3; s->fp[fb][f] = m; m += s->N3; s->fa[fb][f] = m; m += s->N3;
            }
    if (real)
        for (int c = 0; c < 3; c++) { s->mis[c] = m; m += s->N3; s->hq[c] = m; m += s->N3; }
    /* column order -> packed slots (the real mode: 12 columns, imaginary parts zero) */
    size_t bytes = s->N3 * sizeof(double);
    if (real) {
        for (int a = 0; a < 3; a++) {
            memcpy(s->q[U0 + a], cols[0 + a], bytes);  memcpy(s->q[TU0 + a], cols[3 + a], bytes);
            memcpy(s->p[U0 + a], cols[6 + a], bytes);  memcpy(s->p[TU0 + a], cols[9 + a], bytes);
        }
        forces(s);
        return s;
    }
    for (int a = 0; a < 3; a++) {
        memcpy(s->q[U0 + a], cols[0 + a], bytes);  memcpy(s->q[TU0 + a], cols[3 + a], bytes);
        memcpy(s->p[U0 + a], cols[6 + a], bytes);  memcpy(s->p[TU0 + a], cols[9 + a], bytes);
        memcpy(s->q[V0 + a], cols[12 + a], bytes); memcpy(s->q[TV0 + a], cols[15 + a], bytes);
        memcpy(s->p[V0 + a], cols[18 + a], bytes); memcpy(s->p[TV0 + a], cols[21 + a], bytes);
        if (p->gauge) { memcpy(s->th[a], cols[24 + a], bytes); memcpy(s->E[a], cols[27 + a], bytes); }
    }
    /* the start-up of main (scp_sim.c:2802-2836): Higgs start value, fabrics
     * (mf_post_init: Q is C under the lock), net charge, Gauss projections */
    if (higgs) {
        const int N = p->N;
        const long NN = (long)N * N;
        for (long idx = 0; idx < s->N3; idx++) {
            double h = p->higgs_v;
            if (p->higgs_rvoid > 0.0) {
                int i = (int)(idx / NN), j = (int)((idx / N) % N), k = (int)(idx % N);
                double x = -p->L + i * p->dx, y = -p->L + j * p->dx, z = -p->L + k * p->dx;
                double r = sqrt(x * x + y * y + z * z);
                h = p->higgs_v * 0.5 * (1.0 + tanh((r - p->higgs_rvoid) / 0.6));
            }
            s->H[idx] = h;
            s->HV[idx] = 0.0;
        }
    }
    if (mf) {
        fabric_in(s, 1, cols + 54);
        if (p->mf_lock) lock_copy(s);
        else fabric_in(s, 0, cols + 30);
    }
    if (p->gauge) {
        if (p->bc_type == 2 && !net_charge_ok(s)) { orc_free(s); *status = -2; return NULL; }
        if (project) {
            int rc = gauss_project(s);
            if (!rc && g2on) rc = gauss2_project(s);
            if (rc) { orc_free(s); *status = rc; return NULL; }
        }
    }
    forces(s);
    return s;
}

void orc_free(orc_state *s) {
    if (!s) return;
    free(s->mem);
    free(s);
}

void orc_get(const orc_state *s, double *const *cols) {
    size_t bytes = s->N3 * sizeof(double);
    if (s->real) {
        for (int a = 0; a < 3; a++) {
            memcpy(cols[0 + a], s->q[U0 + a], bytes);  memcpy(cols[3 + a], s->q[TU0 + a], bytes);
            memcpy(cols[6 + a], s->p[U0 + a], bytes);  memcpy(cols[9 + a], s->p[TU0 + a], bytes);
        }
        return;
    }
    for (int a = 0; a < 3; a++) {
        memcpy(cols[0 + a], s->q[U0 + a], bytes);  memcpy(cols[3 + a], s->q[TU0 + a], bytes);
        memcpy(cols[6 + a], s->p[U0 + a], bytes);  memcpy(cols[9 + a], s->p[TU0 + a], bytes);
        memcpy(cols[12 + a], s->q[V0 + a], bytes); memcpy(cols[15 + a], s->q[TV0 + a], bytes);
        memcpy(cols[18 + a], s->p[V0 + a], bytes); memcpy(cols[21 + a], s->p[TV0 + a], bytes);
        if (s->P.gauge) { memcpy(cols[24 + a], s->th[a], bytes); memcpy(cols[27 + a], s->E[a], bytes); }
        if (s->g2on) { memcpy(cols[30 + a], s->th2[a], bytes); memcpy(cols[33 + a], s->E2[a], bytes); }
        if (s->mf) {   /* fabric L after C, the complex column order */
            double *const *L = cols + 30;
            memcpy(L[0 + a], s->fq[1][U0 + a], bytes);  memcpy(L[3 + a], s->fq[1][TU0 + a], bytes);
            memcpy(L[6 + a], s->fp[1][U0 + a], bytes);  memcpy(L[9 + a], s->fp[1][TU0 + a], bytes);
            memcpy(L[12 + a], s->fq[1][V0 + a], bytes); memcpy(L[15 + a], s->fq[1][TV0 + a], bytes);
            memcpy(L[18 + a], s->fp[1][V0 + a], bytes); memcpy(L[21 + a], s->fp[1][TV0 + a], bytes);
        }
    }
}

double orc_g_offset(const orc_state *s) { return s->G_offset; }
int orc_cg_iterations(const orc_state *s) { return s->cg_iters; }

void orc_accelerations(orc_state *s, double *const *acc) {
    forces(s);
    size_t bytes = s->N3 * sizeof(double);
    for (int a = 0; a < 3; a++) {
        memcpy(acc[0 + a], s->a[U0 + a], bytes);  memcpy(acc[3 + a], s->a[TU0 + a], bytes);
        memcpy(acc[6 + a], s->a[V0 + a], bytes);  memcpy(acc[9 + a], s->a[TV0 + a], bytes);
        if (s->P.gauge) memcpy(acc[12 + a], s->K[a], bytes);
        else memset(acc[12 + a], 0, bytes);
    }
}

/* do_test_gauge_xform, scp_sim.c:2461-2556 */
double orc_gauge_xform_test(orc_state *s, double *rel_out10) {
    if (!s->P.gauge) return -1.0;
    const int N = s->P.N;
    const long N3 = s->N3;
    const double GG = s->P.g;
    forces(s);
    double *bf = malloc(10 * N3 * sizeof(double)), *alpha = malloc(N3 * sizeof(double));
    if (!bf || !alpha) { free(bf); free(alpha); return -1.0; }
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        for (int a = 0; a < 3; a++) {
            bf[a * N3 + idx] = s->a[U0 + a][idx] * s->a[U0 + a][idx] + s->a[V0 + a][idx] * s->a[V0 + a][idx];
            bf[(3 + a) * N3 + idx] = s->a[TU0 + a][idx] * s->a[TU0 + a][idx]
                                   + s->a[TV0 + a][idx] * s->a[TV0 + a][idx];
            bf[(6 + a) * N3 + idx] = s->K[a][idx];
        }
        bf[9 * N3 + idx] = gauss_at(s, idx, &n);
        uint64_t g = (uint64_t)idx * 6364136223846793005ULL + 1442695040888963407ULL;
        g = g * 6364136223846793005ULL + 1442695040888963407ULL;
        alpha[idx] = (((double)(g >> 11)) / 9007199254740992.0 - 0.5) * 20.0;
    }
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < N3; idx++) {
        nbr_t n = nbrs(N, idx);
        long np[3] = {n.ip, n.jp, n.kp};
        double ca = cos(GG * alpha[idx]), sa = sin(GG * alpha[idx]);
        for (int a = 0; a < 3; a++) {
            double *pairs[4][2] = {{s->q[U0 + a], s->q[V0 + a]}, {s->p[U0 + a], s->p[V0 + a]},
                                   {s->q[TU0 + a], s->q[TV0 + a]}, {s->p[TU0 + a], s->p[TV0 + a]}};
            for (int w = 0; w < 4; w++) {
                double u = pairs[w][0][idx], v = pairs[w][1][idx];
                pairs[w][0][idx] = ca * u + sa * v;
                pairs[w][1][idx] = ca * v - sa * u;
            }
        }
        for (int d = 0; d < 3; d++) s->th[d][idx] = wrap_angle(s->th[d][idx] + GG * (alpha[np[d]] - alpha[idx]));
    }
    forces(s);
    double worst = 0;
    for (int qn = 0; qn < 10; qn++) {
        double sc = 0, dm = 0;
        for (long idx = 0; idx < N3; idx++) {
            nbr_t n = nbrs(N, idx);
            double after;
            if (qn < 3) after = s->a[U0 + qn][idx] * s->a[U0 + qn][idx] + s->a[V0 + qn][idx] * s->a[V0 + qn][idx];
            else if (qn < 6) after = s->a[TU0 + qn - 3][idx] * s->a[TU0 + qn - 3][idx]
                                   + s->a[TV0 + qn - 3][idx] * s->a[TV0 + qn - 3][idx];
            else if (qn < 9) after = s->K[qn - 6][idx];
            else after = gauss_at(s, idx, &n);
            double b0 = bf[qn * N3 + idx];
            if (fabs(b0) > sc) sc = fabs(b0);
            double d = fabs(after - b0);
            if (d > dm) dm = d;
        }
        double rel = dm / fmax(sc, 1.0);
        if (rel_out10) rel_out10[qn] = rel;
        if (rel > worst) worst = rel;
    }
    free(bf);
    free(alpha);
    return worst;
}

int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
