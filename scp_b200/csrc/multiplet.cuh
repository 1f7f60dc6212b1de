// multiplet.cuh -- the covariant stencil of one complex Cosserat matter
// multiplet (Phi_a = u_a + i v_a, Theta_a = tu_a + i tv_a, a = 0, 1, 2) on the
// plane ring, and the plaquette staples of a set of compact link angles.
//
// A matter field is parallel-transported along every link before it is
// differenced.  For direction d with the link phase P at x (link x -> x+d)
// and M at x - d (link x-d -> x):
//     forward   T+ = e^{iP} f(x + d)            (u' = cP u - sP v, v' = cP v + sP u)
//     backward  T- = e^{-iM} f(x - d)           (u' = cM u + sM v, v' = cM v - sM u)
// The covariant Laplacian is (sum_d T+ + T- - 6 f) / dx^2, the covariant
// central difference D_d f = (T+ - T-) / (2 dx), and curl_c = D_{c+1} f_{c+2}
// - D_{c+2} f_{c+1} (indices mod 3).  The lattice current along d is
//     J_d = (1/dx) sum_a Im[f_a^* T+_a]  over Phi and Theta,
// less (eta/2)(T12 - T21), the cross term of the Cosserat coupling, which
// pairs Theta_{d+1} with Phi_{d+2} transported forward and Theta_{d+1}(x+d)
// with Phi_{d+2}(x) transported back (and the same with d+1, d+2 swapped).
// This is the force of compute_forces_complex_gauge (sfa/sim/scp_sim.c:
// 1112-1262) and of the per-fabric force_fabric_gauged_accum (:1292-1381),
// evaluated here one direction at a time so only the running sums stay live.
//
// The link phases come from a policy object: `links(d, cP, sP, cM, sM, cW, sW)`
// fills the forward and backward phase of each component a for direction d,
// and the phase (cW, sW) of the forward link used by the cross term.
#pragma once
#include "ring.cuh"
#include "trig.cuh"

namespace scp {

// field slots inside a multiplet: u_a, v_a, tu_a, tv_a
enum : int { MU = 0, MV = 3, MTU = 6, MTV = 9 };

struct MultipletOut {
    double lsum[12];   // sum over d of forward + backward transports, per field slot
    double curlP[6];   // curl of Phi: [0..2] real part, [3..5] imaginary part
    double curlT[6];   // curl of Theta
    double jlat[3];    // lattice current per direction, cross term included
    double jw[3];      // sum_a w_a Im[f_a^* T+_a] per direction (weighted current, no cross term)
};

// offset of direction d (0: i, 1: j, 2: k) scaled by s
template <class V>
__device__ __forceinline__ double nb(const V &v, int f, int d, int s) {
    return v.at(f, d == 0 ? s : 0, d == 1 ? s : 0, d == 2 ? s : 0);
}

template <bool WEIGHTED, class V, class LinkFn>
__device__ __forceinline__ void covariant_multiplet(const V &v, int base, const double own[12], LinkFn links,
                                                    const double w[3], double idx1, double inva, double eta,
                                                    MultipletOut &o) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double cP[3], sP[3], cM[3], sM[3], cW, sW;
        links(d, cP, sP, cM, sM, cW, sW);
        double fwdRe[3], fwdIm[3];   // Phi_a transported from x + d
        double rawTu[3], rawTv[3];   // Theta_a at x + d, untransported
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const int a = q % 3;
            const int re = base + (q < 3 ? MU : MTU) + a, im = base + (q < 3 ? MV : MTV) + a;
            const double up = nb(v, re, d, 1), vp = nb(v, im, d, 1);
            const double um = nb(v, re, d, -1), vm = nb(v, im, d, -1);
            const double fr = cP[a] * up - sP[a] * vp, fi = cP[a] * vp + sP[a] * up;
            const double br = cM[a] * um + sM[a] * vm, bi = cM[a] * vm - sM[a] * um;
            const int sr = (q < 3 ? MU : MTU) + a, si = (q < 3 ? MV : MTV) + a;
            if (d == 0) { o.lsum[sr] = fr + br; o.lsum[si] = fi + bi; }
            else { o.lsum[sr] = o.lsum[sr] + fr + br; o.lsum[si] = o.lsum[si] + fi + bi; }
            // central differences feeding the curl of this field: component a
            // enters curl_{d+2} with + sign when a = d+1, curl_{d+1} with - when
            // a = d+2; the two directions of one curl component meet in one
            // subtraction, whichever comes first in d
            if (a != d) {
                const double dr = (fr - br) * idx1, di = (fi - bi) * idx1;
                double *cr = q < 3 ? o.curlP : o.curlT;
                const bool plus = (a == (d + 1) % 3);
                const int c = plus ? (d + 2) % 3 : (d + 1) % 3;
                const int other = plus ? (c + 2) % 3 : (c + 1) % 3;   // the direction of the other term
                if (d < other) { cr[c] = dr; cr[3 + c] = di; }
                else if (plus) { cr[c] = dr - cr[c]; cr[3 + c] = di - cr[3 + c]; }
                else { cr[c] = cr[c] - dr; cr[3 + c] = cr[3 + c] - di; }
            }
            if (q < 3) { fwdRe[a] = fr; fwdIm[a] = fi; }
            else { rawTu[a] = up; rawTv[a] = vp; }
        }
        // current: Im[f^* T+] = u Im T+ - v Re T+, Phi then Theta per component
        double j = 0.0, jw = 0.0;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double tfi = cP[a] * rawTv[a] + sP[a] * rawTu[a];
            const double tfr = cP[a] * rawTu[a] - sP[a] * rawTv[a];
            const double jp = own[MU + a] * fwdIm[a] - own[MV + a] * fwdRe[a];
            const double jt = own[MTU + a] * tfi - own[MTV + a] * tfr;
            j += jp;
            j += jt;
            if (WEIGHTED) {
                jw += w[a] * jp;
                jw += w[a] * jt;
            }
        }
        // cross term: Theta_{e} with Phi_{f} for (e, f) = (d+1, d+2) and (d+2, d+1)
        const int e1 = (d + 1) % 3, e2 = (d + 2) % 3;
        const double bR2 = cW * own[MU + e2] + sW * own[MV + e2], bI2 = cW * own[MV + e2] - sW * own[MU + e2];
        const double bR1 = cW * own[MU + e1] + sW * own[MV + e1], bI1 = cW * own[MV + e1] - sW * own[MU + e1];
        const double x12 = (own[MTU + e1] * fwdIm[e2] - own[MTV + e1] * fwdRe[e2]) + (rawTu[e1] * bI2 - rawTv[e1] * bR2);
        const double x21 = (own[MTU + e2] * fwdIm[e1] - own[MTV + e2] * fwdRe[e1]) + (rawTu[e2] * bI1 - rawTv[e2] * bR1);
        o.jlat[d] = inva * j - 0.5 * eta * (x12 - x21);
        if (WEIGHTED) o.jw[d] = jw;
    }
}

// sine of the plaquette of plane (a, b) = (q, q+1 mod 3) at the site offset
// (di, dj, dk) from this thread's: th_a(y) + th_b(y+a) - th_a(y+b) - th_b(y)
template <class V>
__device__ __forceinline__ double plaquette_sin(const V &v, int fth, int q, int di, int dj, int dk) {
    const int a = q, b = (q + 1) % 3;
    const double tay = v.at(fth + a, di, dj, dk), tby = v.at(fth + b, di, dj, dk);
    const double tb_ya = v.at(fth + b, di + (a == 0), dj + (a == 1), dk + (a == 2));
    const double ta_yb = v.at(fth + a, di + (b == 0), dj + (b == 1), dk + (b == 2));
    return sin_bounded(tay + tb_ya - ta_yb - tby);
}

// the plaquette term of the field kick along each direction (compute_forces_
// complex_gauge's staples, sfa/sim/scp_sim.c:1214-1220): differences of the
// plaquette sines of the two planes containing the direction, at x and at x
// less the other direction of the plane.  pim[0..1]: the (0,1) and (2,0)
// sines at x - i, which the caller may carry from the previous plane.
template <class V>
__device__ __forceinline__ void staples(const V &v, int fth, const double pim[2], double st[3], double pat[2]) {
    const double p0 = plaquette_sin(v, fth, 0, 0, 0, 0), p1 = plaquette_sin(v, fth, 1, 0, 0, 0);
    const double p2 = plaquette_sin(v, fth, 2, 0, 0, 0);
    const double p0j = plaquette_sin(v, fth, 0, 0, -1, 0), p1j = plaquette_sin(v, fth, 1, 0, -1, 0);
    const double p1k = plaquette_sin(v, fth, 1, 0, 0, -1), p2k = plaquette_sin(v, fth, 2, 0, 0, -1);
    st[0] = (p0 - p0j) - (p2 - p2k);
    st[1] = -(p0 - pim[0]) + (p1 - p1k);
    st[2] = (p2 - pim[1]) - (p1 - p1j);
    pat[0] = p0;
    pat[1] = p2;
}

}  // namespace scp
