// step_duo.cuh -- the gauged FP64 fused step with two threads per site.
//
// The one-thread-per-site step (step.cuh) needs ~240 registers, which holds
// an SM to eight warps; its time goes to FP64 dependency chains and load
// latency that eight warps cannot cover.  Here every site of the (TX x TY)
// tile has two threads in one CTA of 2*TX*TY:
//   matter thread  (warps 0 .. TY-1)   the three complex Phi fields: their
//                  covariant Laplacians and derivatives, the potential, the
//                  Phi parts of the lattice current and of the Cosserat cross
//                  term, and the Phi kick / drift;
//   theta thread   (warps TY .. 2TY-1) the three complex Theta fields and the
//                  links: Theta Laplacians and derivatives, the Theta parts of
//                  the current, the plaquette staples, and the Theta, E and
//                  link kick / drift.
// Each needs about half the live values, so twice the warps stay resident.
// The couplings between the halves (each curl feeds the other's force, the
// current needs both) go through shared memory between the two phases of a
// plane, with a barrier over the two warps of one tile row (TX = 32: a warp
// is a row).  Both threads evaluate the link cos/sin they transport with.
//
// Arithmetic is that of step_item's gauged F64 branch term by term; the
// current J_d is summed in the same order (Phi_0, Theta_0, Phi_1, ...).
// Staging, work plan and the fused leapfrog scheme are those of step.cuh.
#pragma once
#include "step.cuh"

namespace scp {

template <int TX, int TY>
struct DuoLayout {
    static_assert(TX == 32, "one warp per tile row and role");
    static constexpr int NF = 15;
    static constexpr int PX = TX + 2, PY = TY + 2;
    static constexpr int PLANE = NF * PY * PX;
    static constexpr int NT = TX * TY;                 // sites of a tile
    static constexpr int NHALO = 2 * TX + 2 * TY + 2;
    static constexpr int HPT = (NHALO + NT - 1) / NT;   // halo sites per thread of one role
    // exchange words per site, written in phase 1 and read in phase 2:
    // matter -> theta: curl of Phi (re 3, im 3), Phi current terms (d, a), T12 - T21 (d)
    // theta -> matter: curl of Theta (re 3, im 3); theta's own current terms (d, a)
    // theta -> itself: the staples (kept in shared memory over the barrier)
    static constexpr int X_CRP = 0, X_CIP = 3, X_JP = 6, X_TD = 15, X_CRT = 18, X_CIT = 21, X_JT = 24, X_ST = 33,
                         NX = 36;
    static constexpr size_t ring_bytes = sizeof(double) * 3 * PLANE;
    static constexpr size_t smem_bytes = ring_bytes + sizeof(double) * NX * NT;
};

__device__ __forceinline__ void pair_barrier(int id) {
    asm volatile("bar.sync %0, 64;\n" ::"r"(id) : "memory");
}

template <int TX, int TY, bool FIRST>
__device__ __forceinline__ void duo_item(const StepIO<F64> &io, const StepConsts &c, const Piece &pc,
                                         const bool SYNC, const bool DAMP, double *ring, double *ex) {
    using DL = DuoLayout<TX, TY>;
    constexpr int NT = DL::NT, PX = DL::PX, PY = DL::PY, PLANE = DL::PLANE, FS = PY * PX;
    const int N = c.N;
    const long long N3 = c.N3;
    const int tid = threadIdx.x;
    const int role = tid / NT;   // 0 matter, 1 theta (whole warps)
    const int s = tid - role * NT;
    const int tx = s % TX, ty = s / TX;
    const int k0 = pc.kt * TX, j0 = pc.jt * TY;
    const int i0 = pc.i0, i1 = pc.i1;
    const int nk = min(k0 + TX, N) - k0, nj = min(j0 + TY, N) - j0;
    const bool act = (tx < nk) && (ty < nj);
    const int j = j0 + ty, k = k0 + tx;
    const int oc = j * N + k;
    const int c_s = (ty + 1) * PX + tx + 1;
    const double dt = c.dt, hdt = c.hdt, idx1 = c.idx1, idx2 = c.idx2;
    auto XS = [&](int slot, int f, int r, int col) -> double { return ring[(slot * DL::NF + f) * FS + r * PX + col]; };
    auto EX = [&](int w) -> double & { return ex[w * NT + s]; };

    // halo copies of this thread: edge sites (all of the role's fields) and,
    // for the theta role, the two corners (link angles only)
    int h_s[DL::HPT], h_g[DL::HPT], h_kind[DL::HPT];
    {
        const int jlo = wrapi(j0 - 1, N), jhi = wrapi(j0 + nj, N);
        const int klo = wrapi(k0 - 1, N), khi = wrapi(k0 + nk, N);
#pragma unroll
        for (int q = 0; q < DL::HPT; q++) {
            const int h = s + q * NT;
            int r = 0, col = 0, gj = 0, gk = 0, kind = 0;
            if (h < nk) { r = 0; col = h + 1; gj = jlo; gk = k0 + h; kind = 1; }
            else if (h < 2 * nk) { r = nj + 1; col = h - nk + 1; gj = jhi; gk = k0 + h - nk; kind = 1; }
            else if (h < 2 * nk + nj) { r = h - 2 * nk + 1; col = 0; gj = j0 + h - 2 * nk; gk = klo; kind = 1; }
            else if (h < 2 * nk + 2 * nj) { r = h - 2 * nk - nj + 1; col = nk + 1; gj = j0 + h - 2 * nk - nj; gk = khi; kind = 1; }
            else if (role == 1 && h == 2 * nk + 2 * nj) { r = nj + 1; col = 0; gj = jhi; gk = klo; kind = 2; }
            else if (role == 1 && h == 2 * nk + 2 * nj + 1) { r = 0; col = nk + 1; gj = jlo; gk = khi; kind = 2; }
            h_s[q] = r * PX + col;
            h_g[q] = gj * N + gk;
            h_kind[q] = kind;
        }
    }
    auto issue = [&](int p, int slot) {
        const long long pb = (long long)wrapi(p, N) * N * N;
        double *sb = ring + slot * PLANE;
        const double *gb = io.xin + pb;
        if (role == 0) {
            if (act) {
#pragma unroll
                for (int f = 0; f < FTU; f++) cp_async8(sb + f * FS + c_s, gb + f * N3 + oc);
            }
#pragma unroll
            for (int q = 0; q < DL::HPT; q++) {
                if (h_kind[q] != 1) continue;
#pragma unroll
                for (int f = 0; f < FTU; f++) cp_async8(sb + f * FS + h_s[q], gb + f * N3 + h_g[q]);
            }
        } else {
            if (act) {
#pragma unroll
                for (int f = FTU; f < DL::NF; f++) cp_async8(sb + f * FS + c_s, gb + f * N3 + oc);
            }
#pragma unroll
            for (int q = 0; q < DL::HPT; q++) {
                if (h_kind[q] == 0) continue;
                const int f0 = h_kind[q] == 1 ? FTU : FTH;
#pragma unroll
                for (int f = FTU; f < DL::NF; f++)
                    if (f >= f0) cp_async8(sb + f * FS + h_s[q], gb + f * N3 + h_g[q]);
            }
        }
    };
    // sine of the plaquette angle of plane (a, b) = (q, q+1) at ring position
    // (r, col) of slot sc, the next plane in slot sp (as step_item's plaq_sin)
    auto plaq_sin = [&](int q, int sc, int sp, int r, int col) -> double {
        const int a = q, b = (q + 1) % 3;
        const int sa = (a == 0) ? sp : sc, ra = r + (a == 1 ? 1 : 0), ca = col + (a == 2 ? 1 : 0);
        const int sb = (b == 0) ? sp : sc, rb = r + (b == 1 ? 1 : 0), cb = col + (b == 2 ? 1 : 0);
        return sin_bounded(XS(sc, FTH + a, r, col) + XS(sa, FTH + b, ra, ca) - XS(sb, FTH + a, rb, cb) -
                           XS(sc, FTH + b, r, col));
    };

    __syncthreads();   // the previous item finished reading the ring and the exchange words
    issue(i0 - 1, 0);
    issue(i0, 1);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    // this role's complex fields: matter (u0..2, v0..2) = slots FU.., theta (tu, tv) = FTU..
    const int fr = role == 0 ? FU : FTU, fi = fr + 3;
    double xm[6];   // x(i-1) of the role's six components at this site
#pragma unroll
    for (int a = 0; a < 3; a++) {
        xm[a] = act ? XS(0, fr + a, ty + 1, tx + 1) : 0.0;
        xm[3 + a] = act ? XS(0, fi + a, ty + 1, tx + 1) : 0.0;
    }
    double c0m = 1.0, s0m = 0.0, P0m = 0.0, P2m = 0.0;   // link 0 and plaquettes (0,1), (2,0) at x - i
    if (act) {
        sincos_bounded(XS(0, FTH + 0, ty + 1, tx + 1), &s0m, &c0m);
        if (role == 1) {
            P0m = plaq_sin(0, 0, 1, ty + 1, tx + 1);
            P2m = plaq_sin(2, 0, 1, ty + 1, tx + 1);
        }
    }
    if (i0 + 1 <= i1) issue(i0 + 1, 2);
    cp_async_commit();

    for (int i = i0; i < i1; i++) {
        const int sc = (i - i0 + 1) % 3, sp = (i - i0 + 2) % 3, sn = (i - i0) % 3;
        cp_async_wait<0>();
        __syncthreads();   // planes i-1 (registers), i, i+1 resident; slot sn free; exchange words free
        if (i + 2 <= i1) issue(i + 2, sn);
        cp_async_commit();
        const long long site = (long long)i * N * N + oc;

        // ---- phase 1: transports, Laplacians, curls, current terms
        double fu[3], fv[3];      // this role's centre values
        double lapU[3], lapV[3];  // sums of the transported neighbours
        double w[9];              // momenta: matter 6; theta 6 + E 3
        if (act) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                fu[a] = XS(sc, fr + a, ty + 1, tx + 1);
                fv[a] = XS(sc, fi + a, ty + 1, tx + 1);
            }
            double cr[3], ci[3];   // curl of this role's field (matter: Phi, theta: Theta)
#pragma unroll
            for (int d = 0; d < 3; d++) {
                double cP, sP, cM, sM;
                sincos_bounded(XS(sc, FTH + d, ty + 1, tx + 1), &sP, &cP);
                if (d == 0) { cM = c0m; sM = s0m; c0m = cP; s0m = sP; }
                else if (d == 1) sincos_bounded(XS(sc, FTH + 1, ty, tx + 1), &sM, &cM);
                else sincos_bounded(XS(sc, FTH + 2, ty + 1, tx), &sM, &cM);
                double TRpq[3], TIpq[3];   // forward transports (matter: for the current and T terms)
                double upr[3], vpr[3];     // raw neighbours at x + d (theta: current)
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    double up, vp, um, vm;
                    if (d == 0) {
                        up = XS(sp, fr + q, ty + 1, tx + 1); vp = XS(sp, fi + q, ty + 1, tx + 1);
                        um = xm[q]; vm = xm[3 + q];
                    } else if (d == 1) {
                        up = XS(sc, fr + q, ty + 2, tx + 1); vp = XS(sc, fi + q, ty + 2, tx + 1);
                        um = XS(sc, fr + q, ty, tx + 1);     vm = XS(sc, fi + q, ty, tx + 1);
                    } else {
                        up = XS(sc, fr + q, ty + 1, tx + 2); vp = XS(sc, fi + q, ty + 1, tx + 2);
                        um = XS(sc, fr + q, ty + 1, tx);     vm = XS(sc, fi + q, ty + 1, tx);
                    }
                    const double TRp = cP * up - sP * vp, TIp = cP * vp + sP * up;
                    const double TRm = cM * um + sM * vm, TIm = cM * vm - sM * um;
                    if (d == 0) { lapU[q] = TRp + TRm; lapV[q] = TIp + TIm; }
                    else { lapU[q] = lapU[q] + TRp + TRm; lapV[q] = lapV[q] + TIp + TIm; }
                    if (q != d) {   // covariant curl, built as the directions come in
                        const double DR = (TRp - TRm) * idx1, DI = (TIp - TIm) * idx1;
                        if (q == (d + 1) % 3) {            // plus term of a = d + 2
                            const int a = (d + 2) % 3;
                            if (d < (a + 2) % 3) { cr[a] = DR; ci[a] = DI; }
                            else { cr[a] = DR - cr[a]; ci[a] = DI - ci[a]; }
                        } else {                           // minus term of a = d + 1
                            const int a = (d + 1) % 3;
                            if (d < (a + 1) % 3) { cr[a] = DR; ci[a] = DI; }
                            else { cr[a] = cr[a] - DR; ci[a] = ci[a] - DI; }
                        }
                    }
                    TRpq[q] = TRp; TIpq[q] = TIp;
                    upr[q] = up; vpr[q] = vp;
                }
                if (role == 0) {
                    // Phi current terms and the Cosserat cross term T12 - T21 of link d
                    // (scp_sim.c:1232-1249), with Theta read from the ring
#pragma unroll
                    for (int a = 0; a < 3; a++) EX(DL::X_JP + 3 * d + a) = fu[a] * TIpq[a] - fv[a] * TRpq[a];
                    const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
                    const int rr = ty + 1 + (d == 1 ? 1 : 0), cc = tx + 1 + (d == 2 ? 1 : 0);
                    const int sx = d == 0 ? sp : sc;   // slot of x + d
                    const double WpR1 = cP * fu[d2] + sP * fv[d2], WpI1 = cP * fv[d2] - sP * fu[d2];
                    const double WpR2 = cP * fu[d1] + sP * fv[d1], WpI2 = cP * fv[d1] - sP * fu[d1];
                    const double T12 = (XS(sc, FTU + d1, ty + 1, tx + 1) * TIpq[d2] - XS(sc, FTV + d1, ty + 1, tx + 1) * TRpq[d2])
                                     + (XS(sx, FTU + d1, rr, cc) * WpI1 - XS(sx, FTV + d1, rr, cc) * WpR1);
                    const double T21 = (XS(sc, FTU + d2, ty + 1, tx + 1) * TIpq[d1] - XS(sc, FTV + d2, ty + 1, tx + 1) * TRpq[d1])
                                     + (XS(sx, FTU + d2, rr, cc) * WpI2 - XS(sx, FTV + d2, rr, cc) * WpR2);
                    EX(DL::X_TD + d) = T12 - T21;
                } else {
                    // Theta current terms: transports recomputed from the raw neighbours
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        const double TIt = cP * vpr[a] + sP * upr[a];
                        const double TRt = cP * upr[a] - sP * vpr[a];
                        EX(DL::X_JT + 3 * d + a) = fu[a] * TIt - fv[a] * TRt;
                    }
                }
            }
            if (role == 0) {
#pragma unroll
                for (int a = 0; a < 3; a++) { EX(DL::X_CRP + a) = cr[a]; EX(DL::X_CIP + a) = ci[a]; }
            } else {
#pragma unroll
                for (int a = 0; a < 3; a++) { EX(DL::X_CRT + a) = cr[a]; EX(DL::X_CIT + a) = ci[a]; }
                // staples (scp_sim.c:1214-1220)
                const double P0 = plaq_sin(0, sc, sp, ty + 1, tx + 1), P1 = plaq_sin(1, sc, sp, ty + 1, tx + 1);
                const double P2 = plaq_sin(2, sc, sp, ty + 1, tx + 1);
                const double P0jm = plaq_sin(0, sc, sp, ty, tx + 1), P1jm = plaq_sin(1, sc, sp, ty, tx + 1);
                const double P1km = plaq_sin(1, sc, sp, ty + 1, tx), P2km = plaq_sin(2, sc, sp, ty + 1, tx);
                EX(DL::X_ST + 0) = (P0 - P0jm) - (P2 - P2km);
                EX(DL::X_ST + 1) = -(P0 - P0m) + (P1 - P1km);
                EX(DL::X_ST + 2) = (P2 - P2m) - (P1 - P1jm);
                P0m = P0; P2m = P2;
            }
        }
        pair_barrier(1 + ty);   // both halves of this row's sites have written their words

        // ---- phase 2: forces, kicks, damping, drift
        if (act) {
            if (role == 0) {
#pragma unroll
                for (int f = 0; f < 6; f++) w[f] = __ldg(io.win + (FU + f) * N3 + site);
            } else {
#pragma unroll
                for (int f = 0; f < 9; f++) w[f] = __ldg(io.win + (FTU + f) * N3 + site);
            }
            double dmp = 1.0;
            if (DAMP && !FIRST) {
                const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
                const double r = sqrt(x * x + y * y + z * z);
                const double Rd = c.L - c.damp_width;
                if (r > Rd) {
                    double sc2 = (r - Rd) / c.damp_width;
                    if (sc2 > 1) sc2 = 1;
                    dmp = 1.0 - c.damp_rate * sc2 * sc2;
                }
            }
            bool bad = false;
            auto put = [&](int f, double x, double v, double wn) {
                st_cs(io.xout + f * N3 + site, x);
                io.wout[f * N3 + site] = wn;
                if (SYNC && !FIRST) {
                    st_cs(io.sout + f * N3 + site, v);
                    bad |= !isfinite(x) || !isfinite(v);
                }
            };
            double acc[6];
            if (role == 0) {
                // potential pieces (scp_sim.c:946-958)
                const double s0 = fu[0] * fu[0] + fv[0] * fv[0];
                const double s1 = fu[1] * fu[1] + fv[1] * fv[1];
                const double s2 = fu[2] * fu[2] + fv[2] * fv[2];
                const double sp3 = s0 * s1 * s2;
                const double den = 1.0 + c.kappa * sp3;
                const double Vp = 0.5 * c.mu / (den * den);
                const double rest[3] = {s1 * s2, s0 * s2, s0 * s1};
                const double m2 = c.m2, eta = c.eta;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const double lUP = (lapU[a] - 6.0 * fu[a]) * idx2;
                    const double lVP = (lapV[a] - 6.0 * fv[a]) * idx2;
                    acc[a] = lUP - m2 * fu[a] - 2.0 * Vp * fu[a] * rest[a] + eta * EX(DL::X_CRT + a);
                    acc[3 + a] = lVP - m2 * fv[a] - 2.0 * Vp * fv[a] * rest[a] + eta * EX(DL::X_CIT + a);
                }
            } else {
                const double mt2 = c.mtheta2, eta = c.eta;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const double lUT = (lapU[a] - 6.0 * fu[a]) * idx2;
                    const double lVT = (lapV[a] - 6.0 * fv[a]) * idx2;
                    acc[a] = lUT - mt2 * fu[a] + eta * EX(DL::X_CRP + a);
                    acc[3 + a] = lVT - mt2 * fv[a] + eta * EX(DL::X_CIP + a);
                }
            }
#pragma unroll
            for (int q = 0; q < 6; q++) {
                const int f = (q < 3 ? fr : fi) + q % 3;
                const double x0 = q < 3 ? fu[q] : fv[q - 3];
                double v = FIRST ? w[q] : w[q] + hdt * acc[q];
                if (DAMP && !FIRST) v *= dmp;
                const double wn = v + hdt * acc[q];
                put(f, x0 + dt * wn, v, wn);
            }
            if (role == 1) {
                const double eta = c.eta, gad = c.gad;
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    double Jg = 0.0;
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        Jg += EX(DL::X_JP + 3 * d + a);
                        Jg += EX(DL::X_JT + 3 * d + a);
                    }
                    double K = c.inva * Jg - 0.5 * eta * EX(DL::X_TD + d);
                    K = c.stp * EX(DL::X_ST + d) + c.g * K;
                    double E = FIRST ? w[6 + d] : w[6 + d] + hdt * K;
                    if (DAMP && !FIRST) E *= dmp;
                    const double Eh = E + hdt * K;
                    put(FTH + d, link_wrap(XS(sc, FTH + d, ty + 1, tx + 1) + gad * Eh), E, Eh);
                }
            }
            if (SYNC && bad) atomicOr(io.flag, 1);
#pragma unroll
            for (int a = 0; a < 3; a++) { xm[a] = fu[a]; xm[3 + a] = fv[a]; }
        }
    }
}

template <int TX, int TY, bool FIRST, bool SYNC, bool DAMP>
__global__ void __launch_bounds__(2 * TX * TY, 2) step_duo_kernel(StepIO<F64> io, StepConsts c, TileGrid tg) {
    extern __shared__ __align__(16) double duo_smem[];
    double *ex = duo_smem + DuoLayout<TX, TY>::ring_bytes / sizeof(double);
    for_each_piece(tg, c.N, [&](const Piece &pc) { duo_item<TX, TY, FIRST>(io, c, pc, SYNC, DAMP, duo_smem, ex); });
}

}  // namespace scp
