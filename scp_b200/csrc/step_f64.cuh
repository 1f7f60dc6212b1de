// step_f64.cuh -- fused FP64 leapfrog step for the complex (v66) and gauged
// (v69) Cosserat Q-ball lattice, one launch per time step.
//
// Time integration.  The reference runs kick / drift / force / kick as about
// ten separate sweeps per step (sfa/sim/scp_sim.c:1583-1716, GPU launch
// sequence sfa/sim/scp_sim.cu:2971-3208) and keeps an acceleration array.
// Here the state between launches is (x_{n+1}, w_n) with the half-step
// momentum w_n = v_n + hdt*a_n, and launch n+1 performs, per site,
//     a_{n+1} = F(x_{n+1})                    (stencil of x_{n+1})
//     v_{n+1} = w_n + hdt*a_{n+1}             (reference stage-4 kick)
//     [v_{n+1} *= damp(r)]                    (reference stage 5, bc_type 0)
//     w_{n+1} = v_{n+1} + hdt*a_{n+1}         (next step's stage-1 kick)
//     x_{n+2} = x_{n+1} + dt*w_{n+1}          (next step's drift)
// with the same arithmetic, in the same order, as the reference's sweeps, so
// no acceleration array is stored and each state word is read once and
// written once per step.  Links follow the same pattern with E and the
// wrapped link drift th += -g*dx*dt*E.  The launch that starts a run
// (FIRST) reads v_0 instead of w and skips the stage-4 kick; a SYNC launch
// also stores v_{n+1} and E_{n+1} for diagnostics and snapshots.
//
// Data movement.  Persistent CTAs walk work items = (TX x TY) columns in
// (k, j) times segments of SEG planes in i.  A CTA streams its column plane
// by plane through a 3-slot shared-memory ring (plane i, plane i+1, and
// plane i+2 in flight via cp.async), holding the x(i-1) centre values of its
// own sites in registers.  Halo rows/columns wrap periodically.  In gauged
// mode the link cos/sin and plaquette sines of each plane are computed once
// per site into shared memory (plus the low-side halo row and column that
// the backward transports and staples need) instead of once per use.
#pragma once
#include "common.cuh"

namespace scp {

struct StepIO64 {
    const double *xin;   // NF arrays of N^3: positions x_{n+1}
    double *xout;        // NF arrays: x_{n+2}
    const double *win;   // NF arrays: w_n (or v_0, E_0 when FIRST)
    double *wout;        // NF arrays: w_{n+1} (may alias win)
    double *sout;        // NF arrays: v_{n+1}, E_{n+1} (SYNC only)
    int *flag;           // nonfinite flag (SYNC only)
};

// gauge-quantity slots of the per-plane shared array
enum : int { GQ_C0 = 0, GQ_S0 = 3, GQ_P0 = 6, GQ_N = 9 };

template <int TX, int TY, bool GAUGED>
struct F64Layout {
    static constexpr int NF = GAUGED ? 15 : 12;
    static constexpr int PX = TX + 2, PY = TY + 2;
    static constexpr int PLANE = NF * PY * PX;            // doubles per ring slot
    static constexpr int GX = TX + 1, GY = TY + 1;
    static constexpr int GPLANE = GQ_N * GY * GX;
    static constexpr size_t smem_bytes =
        sizeof(double) * (size_t)(3 * PLANE + (GAUGED ? 2 * GPLANE : 0));
};

template <int TX, int TY, bool GAUGED, bool FIRST, bool SYNC, bool DAMP>
__global__ void __launch_bounds__(TX * TY)
step_f64_kernel(StepIO64 io, StepConsts c, TileGrid tg) {
    using LY = F64Layout<TX, TY, GAUGED>;
    constexpr int NF = LY::NF, PX = LY::PX, PY = LY::PY;
    extern __shared__ double smem[];
    double *xs = smem;                         // [3][NF][PY][PX]
    double *gq = smem + 3 * LY::PLANE;         // [2][GQ_N][GY][GX]
    auto XS = [&](int slot, int f, int r, int col) -> double & {
        return xs[((slot * NF + f) * PY + r) * PX + col];
    };
    auto GQ = [&](int slot, int q, int r, int col) -> double & {
        return gq[((slot * GQ_N + q) * LY::GY + r) * LY::GX + col];
    };

    const int N = c.N;
    const long long N3 = c.N3;
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;

    for (int item = blockIdx.x; item < tg.nitems; item += gridDim.x) {
        const int kt = item % tg.ntx;
        const int jt = (item / tg.ntx) % tg.nty;
        const int sg = item / (tg.ntx * tg.nty);
        const int k0 = kt * TX, j0 = jt * TY;
        const int i0 = sg * tg.seg, i1 = min(i0 + tg.seg, N);
        const int k = k0 + tx, j = j0 + ty;
        const int kl = min(k0 + TX, N) - 1, jl = min(j0 + TY, N) - 1;   // last valid in tile
        const bool act = (k < N) && (j < N);

        // global in-plane offsets of the sites this thread copies into the ring
        const long long oc = (long long)j * N + k;
        const int jlo = wrapi(j0 - 1, N), jhi = wrapi(jl + 1, N);
        const int klo = wrapi(k0 - 1, N), khi = wrapi(kl + 1, N);
        const bool ld_rlo = act && ty == 0, ld_rhi = act && j == jl;
        const bool ld_clo = act && tx == 0, ld_chi = act && k == kl;

        auto issue_plane = [&](int p, int slot) {
            const int ip = wrapi(p, N);
            const long long pb = (long long)ip * N * N;
            for (int f = 0; f < NF; f++) {
                const double *src = io.xin + (long long)f * N3 + pb;
                if (act) cp_async8(&XS(slot, f, ty + 1, tx + 1), src + oc);
                if (ld_rlo) cp_async8(&XS(slot, f, 0, tx + 1), src + (long long)jlo * N + k);
                if (ld_rhi) cp_async8(&XS(slot, f, ty + 2, tx + 1), src + (long long)jhi * N + k);
                if (ld_clo) cp_async8(&XS(slot, f, ty + 1, 0), src + (long long)j * N + klo);
                if (ld_chi) cp_async8(&XS(slot, f, ty + 1, tx + 2), src + (long long)j * N + khi);
            }
            if (GAUGED) {   // diagonal corners used by the plaquettes of the halo sites
                for (int f = FTH; f < NF; f++) {
                    const double *src = io.xin + (long long)f * N3 + pb;
                    if (act && j == jl && tx == 0)
                        cp_async8(&XS(slot, f, ty + 2, 0), src + (long long)jhi * N + klo);
                    if (act && ty == 0 && k == kl)
                        cp_async8(&XS(slot, f, 0, tx + 2), src + (long long)jlo * N + khi);
                }
            }
        };

        // gauge quantities of plane in slot sc (next plane in slot sp) into gq slot gs
        auto gauge_plane = [&](int sc, int sp, int gs) {
            constexpr int NS = LY::GY * LY::GX;
            for (int s = threadIdx.x; s < NS; s += TX * TY) {
                const int r = s / LY::GX, col = s % LY::GX;
                if ((r == 0 && col == 0) || r > jl - j0 + 1 || col > kl - k0 + 1) continue;
                const double t0 = XS(sc, FTH + 0, r, col), t1 = XS(sc, FTH + 1, r, col);
                const double t2 = XS(sc, FTH + 2, r, col);
                double sn, cs;
                if (r > 0 && col > 0) {
                    sincos(t0, &sn, &cs); GQ(gs, GQ_C0 + 0, r, col) = cs; GQ(gs, GQ_S0 + 0, r, col) = sn;
                }
                if (col > 0) {
                    sincos(t1, &sn, &cs); GQ(gs, GQ_C0 + 1, r, col) = cs; GQ(gs, GQ_S0 + 1, r, col) = sn;
                }
                if (r > 0) {
                    sincos(t2, &sn, &cs); GQ(gs, GQ_C0 + 2, r, col) = cs; GQ(gs, GQ_S0 + 2, r, col) = sn;
                }
                // plaquette angle th_a(y) + th_b(y+a) - th_a(y+b) - th_b(y), planes (0,1) (1,2) (2,0)
                if (col > 0)
                    GQ(gs, GQ_P0 + 0, r, col) = sin(t0 + XS(sp, FTH + 1, r, col) - XS(sc, FTH + 0, r + 1, col) - t1);
                GQ(gs, GQ_P0 + 1, r, col) = sin(t1 + XS(sc, FTH + 2, r + 1, col) - XS(sc, FTH + 1, r, col + 1) - t2);
                if (r > 0)
                    GQ(gs, GQ_P0 + 2, r, col) = sin(t2 + XS(sc, FTH + 0, r, col + 1) - XS(sp, FTH + 2, r, col) - t0);
            }
        };

        __syncthreads();   // previous item finished reading the ring
        // prologue: planes i0-1 and i0, then plane i0+1 in flight
        issue_plane(i0 - 1, 0);
        issue_plane(i0, 1);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        double xm[12];     // x(i-1) at this thread's site, matter fields
#pragma unroll
        for (int f = 0; f < 12; f++) xm[f] = act ? XS(0, f, ty + 1, tx + 1) : 0.0;
        if (GAUGED) gauge_plane(0, 1, 1);
        issue_plane(i0 + 1, 2);
        cp_async_commit();

        for (int i = i0; i < i1; i++) {
            const int sc = (i - i0 + 1) % 3, sp = (i - i0 + 2) % 3, sn = (i - i0) % 3;
            const int gs = (i - i0) & 1, gm = gs ^ 1;
            cp_async_wait<0>();
            __syncthreads();
            if (i + 2 <= i1) issue_plane(i + 2, sn);
            cp_async_commit();
            const long long site = (long long)i * N * N + oc;
            double w[NF];
            if (act) {
#pragma unroll
                for (int f = 0; f < NF; f++) w[f] = __ldg(io.win + (long long)f * N3 + site);
            }
            if (GAUGED) {
                gauge_plane(sc, sp, gs);
                __syncthreads();
            }
            if (!act) continue;

            double acc[12];
            double K[3] = {0.0, 0.0, 0.0};
            double ctr[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) ctr[f] = XS(sc, f, ty + 1, tx + 1);
            // potential pieces (scp_sim.c:946-958)
            const double s0 = ctr[FU + 0] * ctr[FU + 0] + ctr[FV + 0] * ctr[FV + 0];
            const double s1 = ctr[FU + 1] * ctr[FU + 1] + ctr[FV + 1] * ctr[FV + 1];
            const double s2 = ctr[FU + 2] * ctr[FU + 2] + ctr[FV + 2] * ctr[FV + 2];
            const double sp3 = s0 * s1 * s2;
            const double den = 1.0 + c.kappa * sp3;
            const double Vp = 0.5 * c.mu / (den * den);
            const double rest[3] = {s1 * s2, s0 * s2, s0 * s1};

            if (!GAUGED) {
                // compute_forces_complex, scp_sim.c:931-994
                auto nb = [&](int f, int which) -> double {   // 0 ip 1 im 2 jp 3 jm 4 kp 5 km
                    switch (which) {
                        case 0: return XS(sp, f, ty + 1, tx + 1);
                        case 1: return xm[f];
                        case 2: return XS(sc, f, ty + 2, tx + 1);
                        case 3: return XS(sc, f, ty, tx + 1);
                        case 4: return XS(sc, f, ty + 1, tx + 2);
                        default: return XS(sc, f, ty + 1, tx);
                    }
                };
                auto lap = [&](int f) -> double {
                    return (nb(f, 0) + nb(f, 1) + nb(f, 2) + nb(f, 3) + nb(f, 4) + nb(f, 5) - 6.0 * ctr[f]) * c.idx2;
                };
                auto curl = [&](int g0, int a) -> double {
                    if (a == 0) return (nb(g0 + 2, 2) - nb(g0 + 2, 3) - nb(g0 + 1, 4) + nb(g0 + 1, 5)) * c.idx1;
                    if (a == 1) return (nb(g0 + 0, 4) - nb(g0 + 0, 5) - nb(g0 + 2, 0) + nb(g0 + 2, 1)) * c.idx1;
                    return (nb(g0 + 1, 0) - nb(g0 + 1, 1) - nb(g0 + 0, 2) + nb(g0 + 0, 3)) * c.idx1;
                };
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    double x = ctr[FU + a];
                    acc[FU + a] = lap(FU + a) - c.m2 * x - 2.0 * Vp * x * rest[a] + c.eta * curl(FTU, a);
                    x = ctr[FV + a];
                    acc[FV + a] = lap(FV + a) - c.m2 * x - 2.0 * Vp * x * rest[a] + c.eta * curl(FTV, a);
                    x = ctr[FTU + a];
                    acc[FTU + a] = lap(FTU + a) - c.mtheta2 * x + c.eta * curl(FU, a);
                    x = ctr[FTV + a];
                    acc[FTV + a] = lap(FTV + a) - c.mtheta2 * x + c.eta * curl(FV, a);
                }
            } else {
                // compute_forces_complex_gauge pass C, scp_sim.c:1112-1262
                // complex fields f=0..2 Phi_a, f=3..5 Theta_a: re slot / im slot
                const double fu[6] = {ctr[FU], ctr[FU + 1], ctr[FU + 2], ctr[FTU], ctr[FTU + 1], ctr[FTU + 2]};
                const double fv[6] = {ctr[FV], ctr[FV + 1], ctr[FV + 2], ctr[FTV], ctr[FTV + 1], ctr[FTV + 2]};
                double lapU[6], lapV[6];
                double DcU[3][6], DcV[3][6];
                double TRp_[3][3], TIp_[3][3];   // forward transports of Phi (current)
                double tup[3][3], tvp[3][3];     // raw Theta at x+d (seagull)
                double cPd[3], sPd[3];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    double cP, sP, cM, sM;
                    cP = GQ(gs, GQ_C0 + d, ty + 1, tx + 1);
                    sP = GQ(gs, GQ_S0 + d, ty + 1, tx + 1);
                    if (d == 0) { cM = GQ(gm, GQ_C0, ty + 1, tx + 1); sM = GQ(gm, GQ_S0, ty + 1, tx + 1); }
                    else if (d == 1) { cM = GQ(gs, GQ_C0 + 1, ty, tx + 1); sM = GQ(gs, GQ_S0 + 1, ty, tx + 1); }
                    else { cM = GQ(gs, GQ_C0 + 2, ty + 1, tx); sM = GQ(gs, GQ_S0 + 2, ty + 1, tx); }
                    cPd[d] = cP; sPd[d] = sP;
#pragma unroll
                    for (int q = 0; q < 6; q++) {
                        const int fre = q < 3 ? FU + q : FTU + q - 3;
                        const int fim = q < 3 ? FV + q : FTV + q - 3;
                        double up, vp, um, vm;
                        if (d == 0) {
                            up = XS(sp, fre, ty + 1, tx + 1); vp = XS(sp, fim, ty + 1, tx + 1);
                            um = xm[fre]; vm = xm[fim];
                        } else if (d == 1) {
                            up = XS(sc, fre, ty + 2, tx + 1); vp = XS(sc, fim, ty + 2, tx + 1);
                            um = XS(sc, fre, ty, tx + 1);     vm = XS(sc, fim, ty, tx + 1);
                        } else {
                            up = XS(sc, fre, ty + 1, tx + 2); vp = XS(sc, fim, ty + 1, tx + 2);
                            um = XS(sc, fre, ty + 1, tx);     vm = XS(sc, fim, ty + 1, tx);
                        }
                        const double TRp = cP * up - sP * vp, TIp = cP * vp + sP * up;
                        const double TRm = cM * um + sM * vm, TIm = cM * vm - sM * um;
                        if (d == 0) { lapU[q] = TRp + TRm; lapV[q] = TIp + TIm; }
                        else { lapU[q] = lapU[q] + TRp + TRm; lapV[q] = lapV[q] + TIp + TIm; }
                        DcU[d][q] = (TRp - TRm) * c.idx1;
                        DcV[d][q] = (TIp - TIm) * c.idx1;
                        if (q < 3) { TRp_[d][q] = TRp; TIp_[d][q] = TIp; }
                        else { tup[d][q - 3] = up; tvp[d][q - 3] = vp; }
                        if (q >= 3) { /* theta transports feed the current below */ }
                    }
                    // lattice current J (scp_sim.c:1232-1249), Theta transports recomputed
                    // from the cached raw neighbours to keep the live set small
                    double Jg = 0.0;
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        Jg += fu[a] * TIp_[d][a] - fv[a] * TRp_[d][a];
                        const double TIt = cP * tvp[d][a] + sP * tup[d][a];
                        const double TRt = cP * tup[d][a] - sP * tvp[d][a];
                        Jg += fu[3 + a] * TIt - fv[3 + a] * TRt;
                    }
                    const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
                    const double WpR1 = cP * fu[d2] + sP * fv[d2], WpI1 = cP * fv[d2] - sP * fu[d2];
                    const double WpR2 = cP * fu[d1] + sP * fv[d1], WpI2 = cP * fv[d1] - sP * fu[d1];
                    const double T12 = (fu[3 + d1] * TIp_[d][d2] - fv[3 + d1] * TRp_[d][d2])
                                     + (tup[d][d1] * WpI1 - tvp[d][d1] * WpR1);
                    const double T21 = (fu[3 + d2] * TIp_[d][d1] - fv[3 + d2] * TRp_[d][d1])
                                     + (tup[d][d2] * WpI2 - tvp[d][d2] * WpR2);
                    K[d] = c.inva * Jg - 0.5 * c.eta * (T12 - T21);   // Jlat, staple added below
                }
                // staples (scp_sim.c:1214-1220)
                const double P0 = GQ(gs, GQ_P0 + 0, ty + 1, tx + 1), P1 = GQ(gs, GQ_P0 + 1, ty + 1, tx + 1);
                const double P2 = GQ(gs, GQ_P0 + 2, ty + 1, tx + 1);
                const double st0 = (P0 - GQ(gs, GQ_P0 + 0, ty, tx + 1)) - (P2 - GQ(gs, GQ_P0 + 2, ty + 1, tx));
                const double st1 = -(P0 - GQ(gm, GQ_P0 + 0, ty + 1, tx + 1)) + (P1 - GQ(gs, GQ_P0 + 1, ty + 1, tx));
                const double st2 = (P2 - GQ(gm, GQ_P0 + 2, ty + 1, tx + 1)) - (P1 - GQ(gs, GQ_P0 + 1, ty, tx + 1));
                K[0] = c.stp * st0 + c.g * K[0];
                K[1] = c.stp * st1 + c.g * K[1];
                K[2] = c.stp * st2 + c.g * K[2];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const int d1 = (a + 1) % 3, d2 = (a + 2) % 3;
                    const double reDxT = DcU[d1][3 + d2] - DcU[d2][3 + d1];
                    const double imDxT = DcV[d1][3 + d2] - DcV[d2][3 + d1];
                    const double reDxP = DcU[d1][d2] - DcU[d2][d1];
                    const double imDxP = DcV[d1][d2] - DcV[d2][d1];
                    const double lUP = (lapU[a] - 6.0 * fu[a]) * c.idx2;
                    const double lVP = (lapV[a] - 6.0 * fv[a]) * c.idx2;
                    const double lUT = (lapU[3 + a] - 6.0 * fu[3 + a]) * c.idx2;
                    const double lVT = (lapV[3 + a] - 6.0 * fv[3 + a]) * c.idx2;
                    acc[FU + a] = lUP - c.m2 * fu[a] - 2.0 * Vp * fu[a] * rest[a] + c.eta * reDxT;
                    acc[FV + a] = lVP - c.m2 * fv[a] - 2.0 * Vp * fv[a] * rest[a] + c.eta * imDxT;
                    acc[FTU + a] = lUT - c.mtheta2 * fu[3 + a] + c.eta * reDxP;
                    acc[FTV + a] = lVT - c.mtheta2 * fv[3 + a] + c.eta * imDxP;
                }
                (void)cPd; (void)sPd;
            }

            // kicks, damping, drift (scp_sim.c:1591-1715, fused)
            double dmp = 1.0;
            if (DAMP && !FIRST) {
                const int ii = i;
                const double x = -c.L + ii * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
                const double r = sqrt(x * x + y * y + z * z);
                const double Rd = c.L - c.damp_width;
                if (r > Rd) {
                    double sc2 = (r - Rd) / c.damp_width;
                    if (sc2 > 1) sc2 = 1;
                    dmp = 1.0 - c.damp_rate * sc2 * sc2;
                }
            }
            bool bad = false;
#pragma unroll
            for (int f = 0; f < 12; f++) {
                double v = FIRST ? w[f] : w[f] + c.hdt * acc[f];
                if (DAMP && !FIRST) v *= dmp;
                const double wn = v + c.hdt * acc[f];
                const double xn = ctr[f] + c.dt * wn;
                st_cs(io.xout + (long long)f * N3 + site, xn);
                io.wout[(long long)f * N3 + site] = wn;
                if (SYNC && !FIRST) {
                    st_cs(io.sout + (long long)f * N3 + site, v);
                    bad |= !isfinite(xn) || !isfinite(v);
                }
            }
            if (GAUGED) {
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    double E = FIRST ? w[FTH + d] : w[FTH + d] + c.hdt * K[d];
                    if (DAMP && !FIRST) E *= dmp;
                    const double Eh = E + c.hdt * K[d];
                    const double th = wrap_angle(ctr[FTH + d] + c.gad * Eh);
                    st_cs(io.xout + (long long)(FTH + d) * N3 + site, th);
                    io.wout[(long long)(FTH + d) * N3 + site] = Eh;
                    if (SYNC && !FIRST) {
                        st_cs(io.sout + (long long)(FTH + d) * N3 + site, E);
                        bad |= !isfinite(E) || !isfinite(th);
                    }
                }
            }
            if (SYNC && bad) atomicOr(io.flag, 1);
#pragma unroll
            for (int f = 0; f < 12; f++) xm[f] = ctr[f];
        }
    }
}

}  // namespace scp
