// step2.cuh -- the FP32-compensated leapfrog step with two neighbouring sites
// (k, k+1) per thread, computed with the packed FP32 instructions of sm_100
// (vec2.cuh).  Same time integration, state layout and compensated
// bookkeeping as step_item<F32C> in step.cuh; what changes is the work split:
//
//  * a thread owns the site pair (k, k+1), k even, so every field of the pair
//    is one 8-byte word in global and shared memory (one cp.async, one
//    LDS.64, one STG.64 per field and pair; the bf16 low parts of a pair are
//    one 32-bit word);
//  * the arithmetic of both sites is one FFMA2 / FADD2 / FMUL2 stream, which
//    halves the instructions that bound the one-site FP32C kernel;
//  * the k +- 1 neighbours come from the pair itself plus one scalar load.
//
// Requirements: N even (pairs never straddle a row end and every pair is
// 8-byte aligned) and an even tile width.  The host picks this kernel for
// FP32C grids with even N and the one-site kernel otherwise.
//
// Shared-memory ring: [3 slots][NR fields][TY + 2 rows][TX + 4 columns];
// interior sites sit in columns 2..TX+1 so pairs start on even columns, the
// k-1 / k+1 halo columns are 1 and TX+2.
#pragma once
#include "step.cuh"
#include "vec2.cuh"

#ifndef SCP_PAIR_THREADS_PER_SM
#define SCP_PAIR_THREADS_PER_SM 256
#endif

namespace scp {

template <int TX, int TY, bool GAUGED>
struct Step2Layout {
    static_assert(TX % 2 == 0, "site pairs along k need an even tile width");
    static constexpr int NF = GAUGED ? 15 : 12;
    static constexpr int NR = NF + (GAUGED ? 3 : 0);     // ring fields (+ link low parts)
    static constexpr int PX = TX + 4, PY = TY + 2;
    static constexpr int PLANE = NR * PY * PX;
    static constexpr int NT = (TX / 2) * TY;
    static constexpr int NHALO = TX + 2 * TY + (GAUGED ? 2 : 0);   // pair rows + single columns + corners
    static constexpr int HPT = (NHALO + NT - 1) / NT;
    static constexpr size_t smem_bytes = sizeof(float) * (size_t)(3 * PLANE);
    // resident threads per SM the register allocation is sized for
    // (256: up to 255 registers a thread)
    static constexpr int MIN_BLOCKS = (SCP_PAIR_THREADS_PER_SM / NT) > 0 ? SCP_PAIR_THREADS_PER_SM / NT : 1;
};

__device__ __forceinline__ V2 bf16x2_to_v2(uint32_t u) {
    return V2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
}
__device__ __forceinline__ uint32_t v2_to_bf16x2(V2 a) {
    return (uint32_t)f_to_bf16(a.v.x) | ((uint32_t)f_to_bf16(a.v.y) << 16);
}
__device__ __forceinline__ void st_cs2(float *p, V2 a) { __stcs(reinterpret_cast<float2 *>(p), a.v); }

// Link angle drift with the 2 pi wrap, one lane (th, lo: compensated pair).
__device__ __forceinline__ void link_wrap_c(float *th, float *lo) {
    if (fabsf(*th) > 3.0f) {
        const float kq = rintf(*th * 0.159154943091895336f);
        float t1, e1;
        two_sum(*th, -kq * 6.28318548202514648f, &t1, &e1);   // 2 pi (fp32) times |kq| <= 1
        const float l = *lo + e1 + kq * 1.74845553e-7f;        // 2 pi = 6.2831855f - 1.748e-7
        two_sum(t1, l, th, lo);
    }
}

template <int TX, int TY, bool GAUGED, bool FIRST>
__device__ __forceinline__ void step_item2(const StepIO<F32C> &io, const StepConsts &c, const Piece &pc,
                                           const bool SYNC, const bool DAMP, unsigned char *smem_raw) {
    using LY = Step2Layout<TX, TY, GAUGED>;
    constexpr int NF = LY::NF, NR = LY::NR, PX = LY::PX, PY = LY::PY, NT = LY::NT, HX = TX / 2;
    float *xs = reinterpret_cast<float *>(smem_raw);
    auto AT = [&](int slot, int f, int r, int col) -> float * { return xs + ((slot * NR + f) * PY + r) * PX + col; };
    auto S1 = [&](int slot, int f, int r, int col) -> float { return *AT(slot, f, r, col); };
    // a pair starting on an even column: one 8-byte load
    auto S2 = [&](int slot, int f, int r, int col) -> V2 {
        return V2(*reinterpret_cast<const float2 *>(AT(slot, f, r, col)));
    };
    const int N = c.N;
    const long long N3 = c.N3;
    const int tid = threadIdx.x;
    const int tx2 = tid % HX, ty = tid / HX;
    const V2 dt((float)c.dt), hdt((float)c.hdt), idx1((float)c.idx1), idx2((float)c.idx2);
    const V2 dt_lo((float)(c.dt - (double)(float)c.dt)), hdt_lo((float)(c.hdt - (double)(float)c.hdt));

    const int k0 = pc.kt * TX, j0 = pc.jt * TY;
    const int i0 = pc.i0, i1 = pc.i1;
    const int k = k0 + 2 * tx2, j = j0 + ty;
    const int nk = min(k0 + TX, N) - k0, nj = min(j0 + TY, N) - j0;   // nk is even
    const bool act = (2 * tx2 < nk) && (ty < nj);
    const int oc = j * N + k;
    const int jlo = wrapi(j0 - 1, N), jhi = wrapi(j0 + nj, N);
    const int klo = wrapi(k0 - 1, N), khi = wrapi(k0 + nk, N);
    const int hk = nk / 2;
    const int r0 = ty + 1, cc = 2 + 2 * tx2;                            // ring row / column of the pair

    // halo copies of this thread.  kind 1: a pair of the j-1 / j+1 rows (all
    // ring fields); 2: one site of the k-1 / k+1 columns; 3: a corner site
    // (link angles only, for the plaquettes of the neighbour rows)
    int h_s[LY::HPT], h_g[LY::HPT], h_kind[LY::HPT];
#pragma unroll
    for (int q = 0; q < LY::HPT; q++) {
        const int h = tid + q * NT;
        int r = 0, col = 0, gj = 0, gk = 0, kind = 0;
        if (h < hk) { r = 0; col = 2 + 2 * h; gj = jlo; gk = k0 + 2 * h; kind = 1; }
        else if (h < 2 * hk) { r = nj + 1; col = 2 + 2 * (h - hk); gj = jhi; gk = k0 + 2 * (h - hk); kind = 1; }
        else if (h < 2 * hk + nj) { r = h - 2 * hk + 1; col = 1; gj = j0 + h - 2 * hk; gk = klo; kind = 2; }
        else if (h < 2 * hk + 2 * nj) { r = h - 2 * hk - nj + 1; col = nk + 2; gj = j0 + h - 2 * hk - nj; gk = khi; kind = 2; }
        else if (GAUGED && h == 2 * hk + 2 * nj) { r = nj + 1; col = 1; gj = jhi; gk = klo; kind = 3; }
        else if (GAUGED && h == 2 * hk + 2 * nj + 1) { r = 0; col = nk + 2; gj = jlo; gk = khi; kind = 3; }
        h_s[q] = r * PX + col;
        h_g[q] = gj * N + gk;
        h_kind[q] = kind;
    }
    const int c_s = r0 * PX + cc;

    auto issue_plane = [&](int p, int slot) {
        const long long pb = (long long)wrapi(p, N) * N * N;
        float *sbase = xs + slot * LY::PLANE;
        const float *gbase = io.xin + pb;
        if (act) {
#pragma unroll
            for (int f = 0; f < NF; f++) cp_async8(sbase + f * PY * PX + c_s, gbase + f * N3 + oc);
            if constexpr (NR > NF) {
#pragma unroll
                for (int f = NF; f < NR; f++) cp_async8(sbase + f * PY * PX + c_s, io.tloin + pb + (f - NF) * N3 + oc);
            }
        }
#pragma unroll
        for (int q = 0; q < LY::HPT; q++) {
            const int kind = h_kind[q];
            if (kind == 1) {
#pragma unroll
                for (int f = 0; f < NF; f++) cp_async8(sbase + f * PY * PX + h_s[q], gbase + f * N3 + h_g[q]);
                if constexpr (NR > NF) {
#pragma unroll
                    for (int f = NF; f < NR; f++)
                        cp_async8(sbase + f * PY * PX + h_s[q], io.tloin + pb + (f - NF) * N3 + h_g[q]);
                }
            } else if (kind != 0) {
                const int f0 = (kind == 2) ? 0 : FTH;
#pragma unroll
                for (int f = 0; f < NF; f++)
                    if (f >= f0) cp_async4(sbase + f * PY * PX + h_s[q], gbase + f * N3 + h_g[q]);
                if constexpr (NR > NF) {
#pragma unroll
                    for (int f = NF; f < NR; f++)
                        cp_async4(sbase + f * PY * PX + h_s[q], io.tloin + pb + (f - NF) * N3 + h_g[q]);
                }
            }
        }
    };

    // pair at ring column col (odd: two single loads; even: one 8-byte load)
    auto LDP = [&](int slot, int f, int r, int col, bool odd) -> V2 {
        return odd ? V2(S1(slot, f, r, col), S1(slot, f, r, col + 1)) : S2(slot, f, r, col);
    };
    // sine of the plaquette angle of plane (a,b) = (0,1) (1,2) (2,0) [q = 0,1,2]
    // for the pair at ring (r, col) of slot sc, next plane in slot sp; the
    // angle is the sum of hi differences plus the sum of lo differences
    // (compute_forces_complex_gauge pass B, scp_sim.c:1090-1109)
    auto plaq2 = [&](int q, int sc, int sp, int r, int col, bool odd) -> V2 {
        const int a = q, b = (q + 1) % 3;
        const int sa = (a == 0) ? sp : sc, ra = r + (a == 1 ? 1 : 0), ca = col + (a == 2 ? 1 : 0);
        const int sb = (b == 0) ? sp : sc, rb = r + (b == 1 ? 1 : 0), cb = col + (b == 2 ? 1 : 0);
        const bool odda = odd ^ (a == 2), oddb = odd ^ (b == 2);
        const V2 hi = (LDP(sc, FTH + a, r, col, odd) - LDP(sb, FTH + a, rb, cb, oddb)) +
                      (LDP(sa, FTH + b, ra, ca, odda) - LDP(sc, FTH + b, r, col, odd));
        const V2 lo = (LDP(sc, NF + a, r, col, odd) - LDP(sb, NF + a, rb, cb, oddb)) +
                      (LDP(sa, NF + b, ra, ca, odda) - LDP(sc, NF + b, r, col, odd));
        return sin2(hi + lo);
    };

    __syncthreads();   // previous item finished reading the ring
    issue_plane(i0 - 1, 0);
    issue_plane(i0, 1);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    V2 xm[12];          // x(i-1) of this pair, matter fields
#pragma unroll
    for (int f = 0; f < 12; f++) xm[f] = act ? S2(0, f, r0, cc) : V2(0.f);
    // link 0 and the (0,1), (2,0) plaquettes at x - i (carried from plane to plane)
    V2 c0m(1.f), s0m(0.f), P0m(0.f), P2m(0.f);
    if (GAUGED && act) {
        sincos2(S2(0, FTH + 0, r0, cc), &s0m, &c0m);
        P0m = plaq2(0, 0, 1, r0, cc, false);
        P2m = plaq2(2, 0, 1, r0, cc, false);
    }
    issue_plane(i0 + 1, 2);
    cp_async_commit();

    const V2 m2((float)c.m2), mt2((float)c.mtheta2), eta((float)c.eta);
    const V2 nm2(-(float)c.m2), nmt2(-(float)c.mtheta2);

    for (int i = i0; i < i1; i++) {
        const int sc = (i - i0 + 1) % 3, sp = (i - i0 + 2) % 3, sn = (i - i0) % 3;
        cp_async_wait<0>();
        __syncthreads();
        if (i + 2 <= i1) issue_plane(i + 2, sn);
        cp_async_commit();
        if (!act) continue;
        const long long site = (long long)i * N * N + oc;
        if (c.prefetch && i + 1 < i1) {
#pragma unroll
            for (int f = 0; f < NF; f++) prefetch_line_l2(io.win + f * N3 + site + (long long)N * N);
#pragma unroll
            for (int f = 0; f < 12; f++) prefetch_line_l2(io.loin + f * N3 + site + (long long)N * N);
        }
        V2 w[NF];
        uint32_t lo[12];
#pragma unroll
        for (int f = 0; f < NF; f++) w[f] = V2(__ldg(reinterpret_cast<const float2 *>(io.win + f * N3 + site)));
#pragma unroll
        for (int f = 0; f < 12; f++) lo[f] = __ldg(reinterpret_cast<const uint32_t *>(io.loin + f * N3 + site));

        V2 acc[12];
        V2 K[3];
        V2 ctr[NF];
#pragma unroll
        for (int f = 0; f < NF; f++) ctr[f] = S2(sc, f, r0, cc);
        // potential pieces (scp_sim.c:946-958)
        const V2 s0 = fma2(ctr[FU + 0], ctr[FU + 0], ctr[FV + 0] * ctr[FV + 0]);
        const V2 s1 = fma2(ctr[FU + 1], ctr[FU + 1], ctr[FV + 1] * ctr[FV + 1]);
        const V2 s2 = fma2(ctr[FU + 2], ctr[FU + 2], ctr[FV + 2] * ctr[FV + 2]);
        const V2 den = fma2(V2((float)c.kappa), s0 * s1 * s2, V2(1.f));
        const V2 dd = den * den;
        const float hmu = 0.5f * (float)c.mu;
        const V2 Vp2(2.f * (hmu / dd.v.x), 2.f * (hmu / dd.v.y));     // 2 V'
        const V2 vr[3] = {Vp2 * (s1 * s2), Vp2 * (s0 * s2), Vp2 * (s0 * s1)};

        if (!GAUGED) {
            // compute_forces_complex, scp_sim.c:931-994
            auto nb = [&](int f, int which) -> V2 {   // 0 ip 1 im 2 jp 3 jm 4 kp 5 km
                switch (which) {
                    case 0: return S2(sp, f, r0, cc);
                    case 1: return xm[f];
                    case 2: return S2(sc, f, r0 + 1, cc);
                    case 3: return S2(sc, f, r0 - 1, cc);
                    case 4: return V2(ctr[f].v.y, S1(sc, f, r0, cc + 2));
                    default: return V2(S1(sc, f, r0, cc - 1), ctr[f].v.x);
                }
            };
            auto lap = [&](int f) -> V2 {   // neighbour differences: no cancellation against 6*centre
                const V2 x0 = ctr[f];
                return ((((((nb(f, 0) - x0) + (nb(f, 1) - x0)) + (nb(f, 2) - x0)) + (nb(f, 3) - x0)) +
                         (nb(f, 4) - x0)) + (nb(f, 5) - x0)) * idx2;
            };
            auto curl = [&](int g0, int a) -> V2 {
                if (a == 0) return (((nb(g0 + 2, 2) - nb(g0 + 2, 3)) - nb(g0 + 1, 4)) + nb(g0 + 1, 5)) * idx1;
                if (a == 1) return (((nb(g0 + 0, 4) - nb(g0 + 0, 5)) - nb(g0 + 2, 0)) + nb(g0 + 2, 1)) * idx1;
                return (((nb(g0 + 1, 0) - nb(g0 + 1, 1)) - nb(g0 + 0, 2)) + nb(g0 + 0, 3)) * idx1;
            };
#pragma unroll
            for (int a = 0; a < 3; a++) {
                V2 x = ctr[FU + a];
                acc[FU + a] = fma2(eta, curl(FTU, a), fma2(nm2, x, lap(FU + a)) - vr[a] * x);
                x = ctr[FV + a];
                acc[FV + a] = fma2(eta, curl(FTV, a), fma2(nm2, x, lap(FV + a)) - vr[a] * x);
                x = ctr[FTU + a];
                acc[FTU + a] = fma2(eta, curl(FU, a), fma2(nmt2, x, lap(FTU + a)));
                x = ctr[FTV + a];
                acc[FTV + a] = fma2(eta, curl(FV, a), fma2(nmt2, x, lap(FTV + a)));
            }
        } else {
            // compute_forces_complex_gauge pass C, scp_sim.c:1112-1262, fields q = 0..2
            // Phi_a, q = 3..5 Theta_a.  Laplacians accumulate (transported - centre)
            // differences; the covariant curls are built as the directions come in.
            V2 lapU[6], lapV[6];
            V2 crT[3], ciT[3], crP[3], ciP[3];     // curls of Theta (re, im) and of Phi
#pragma unroll
            for (int d = 0; d < 3; d++) {
                V2 cP, sP, cM, sM;                  // link d at x and at x - d (pass A, :1072-1079)
                sincos2(ctr[FTH + d], &sP, &cP);
                if (d == 0) { cM = c0m; sM = s0m; c0m = cP; s0m = sP; }
                else if (d == 1) sincos2(S2(sc, FTH + 1, r0 - 1, cc), &sM, &cM);
                else sincos2(V2(S1(sc, FTH + 2, r0, cc - 1), ctr[FTH + 2].v.x), &sM, &cM);
                const V2 nsP = -sP, nsM = -sM;
                V2 TRpP[3], TIpP[3], tu[3], tv[3];
#pragma unroll
                for (int q = 0; q < 6; q++) {
                    const int fre = q < 3 ? FU + q : FTU + q - 3;
                    const int fim = q < 3 ? FV + q : FTV + q - 3;
                    V2 up, vp, um, vm;
                    if (d == 0) {
                        up = S2(sp, fre, r0, cc); vp = S2(sp, fim, r0, cc);
                        um = xm[fre]; vm = xm[fim];
                    } else if (d == 1) {
                        up = S2(sc, fre, r0 + 1, cc); vp = S2(sc, fim, r0 + 1, cc);
                        um = S2(sc, fre, r0 - 1, cc); vm = S2(sc, fim, r0 - 1, cc);
                    } else {
                        up = V2(ctr[fre].v.y, S1(sc, fre, r0, cc + 2)); vp = V2(ctr[fim].v.y, S1(sc, fim, r0, cc + 2));
                        um = V2(S1(sc, fre, r0, cc - 1), ctr[fre].v.x); vm = V2(S1(sc, fim, r0, cc - 1), ctr[fim].v.x);
                    }
                    const V2 TRp = fma2(cP, up, nsP * vp), TIp = fma2(cP, vp, sP * up);
                    const V2 TRm = fma2(cM, um, sM * vm), TIm = fma2(cM, vm, nsM * um);
                    const V2 cu = ctr[fre], cv = ctr[fim];
                    const V2 dU = (TRp - cu) + (TRm - cu), dV = (TIp - cv) + (TIm - cv);
                    if (d == 0) { lapU[q] = dU; lapV[q] = dV; }
                    else { lapU[q] = lapU[q] + dU; lapV[q] = lapV[q] + dV; }
                    // central covariant differences enter the curls: component a gets
                    // +D[d = a+1][field a+2] - D[d = a+2][field a+1] (indices mod 3)
                    const int qa = q < 3 ? q : q - 3;
                    if (qa != d) {
                        const V2 DR = (TRp - TRm) * idx1, DI = (TIp - TIm) * idx1;
                        V2 *cr = q < 3 ? crP : crT, *ci = q < 3 ? ciP : ciT;
                        if (qa == (d + 1) % 3) {            // plus term of a = d + 2
                            const int a = (d + 2) % 3;
                            if (d < (a + 2) % 3) { cr[a] = DR; ci[a] = DI; }          // minus term comes later
                            else { cr[a] = DR - cr[a]; ci[a] = DI - ci[a]; }
                        } else {                            // minus term of a = d + 1
                            const int a = (d + 1) % 3;
                            if (d < (a + 1) % 3) { cr[a] = DR; ci[a] = DI; }          // plus term comes later
                            else { cr[a] = cr[a] - DR; ci[a] = ci[a] - DI; }
                        }
                    }
                    if (q < 3) { TRpP[q] = TRp; TIpP[q] = TIp; }
                    else { tu[q - 3] = up; tv[q - 3] = vp; }
                }
                // lattice current J (scp_sim.c:1232-1249): u*TI - v*TR written as
                // u*(TI - v) - v*(TR - u), differences of neighbouring values
                V2 Jg(0.f);
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const V2 fu = ctr[FU + a], fv = ctr[FV + a], tu0 = ctr[FTU + a], tv0 = ctr[FTV + a];
                    const V2 TIt = fma2(cP, tv[a], sP * tu[a]);
                    const V2 TRt = fma2(cP, tu[a], nsP * tv[a]);
                    Jg = Jg + (fu * (TIpP[a] - fv) - fv * (TRpP[a] - fu));
                    Jg = Jg + (tu0 * (TIt - tv0) - tv0 * (TRt - tu0));
                }
                const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
                const V2 fu1 = ctr[FU + d1], fv1 = ctr[FV + d1], fu2 = ctr[FU + d2], fv2 = ctr[FV + d2];
                const V2 WpR1 = fma2(cP, fu2, sP * fv2), WpI1 = fma2(cP, fv2, nsP * fu2);
                const V2 WpR2 = fma2(cP, fu1, sP * fv1), WpI2 = fma2(cP, fv1, nsP * fu1);
                const V2 T12 = (ctr[FTU + d1] * TIpP[d2] - ctr[FTV + d1] * TRpP[d2]) +
                               (tu[d1] * WpI1 - tv[d1] * WpR1);
                const V2 T21 = (ctr[FTU + d2] * TIpP[d1] - ctr[FTV + d2] * TRpP[d1]) +
                               (tu[d2] * WpI2 - tv[d2] * WpR2);
                K[d] = fma2(V2((float)c.inva), Jg, V2(-0.5f * (float)c.eta) * (T12 - T21));   // Jlat
            }
            // staples (scp_sim.c:1214-1220)
            const V2 P0 = plaq2(0, sc, sp, r0, cc, false), P1 = plaq2(1, sc, sp, r0, cc, false);
            const V2 P2 = plaq2(2, sc, sp, r0, cc, false);
            const V2 P0jm = plaq2(0, sc, sp, r0 - 1, cc, false), P1jm = plaq2(1, sc, sp, r0 - 1, cc, false);
            const V2 P1km = plaq2(1, sc, sp, r0, cc - 1, true), P2km = plaq2(2, sc, sp, r0, cc - 1, true);
            const V2 st0 = (P0 - P0jm) - (P2 - P2km);
            const V2 st1 = (P1 - P1km) - (P0 - P0m);
            const V2 st2 = (P2 - P2m) - (P1 - P1jm);
            P0m = P0; P2m = P2;                      // x - i of the next plane
            const V2 stp((float)c.stp), gg((float)c.g);
            K[0] = fma2(stp, st0, gg * K[0]);
            K[1] = fma2(stp, st1, gg * K[1]);
            K[2] = fma2(stp, st2, gg * K[2]);
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const V2 fu = ctr[FU + a], fv = ctr[FV + a];
                acc[FU + a] = fma2(eta, crT[a], fma2(nm2, fu, lapU[a] * idx2) - vr[a] * fu);
                acc[FV + a] = fma2(eta, ciT[a], fma2(nm2, fv, lapV[a] * idx2) - vr[a] * fv);
                acc[FTU + a] = fma2(eta, crP[a], fma2(nmt2, ctr[FTU + a], lapU[3 + a] * idx2));
                acc[FTV + a] = fma2(eta, ciP[a], fma2(nmt2, ctr[FTV + a], lapV[3 + a] * idx2));
            }
        }

        // kicks, damping, drift (scp_sim.c:1591-1715, fused)
        V2 dmp(1.f);
        if (DAMP && !FIRST) {
            const double x = -c.L + i * c.dx, y = -c.L + j * c.dx;
            const double Rd = c.L - c.damp_width;
            float dm[2];
#pragma unroll
            for (int l = 0; l < 2; l++) {
                const double z = -c.L + (k + l) * c.dx;
                const double r = sqrt(x * x + y * y + z * z);
                dm[l] = 1.f;
                if (r > Rd) {
                    double sc2 = (r - Rd) / c.damp_width;
                    if (sc2 > 1) sc2 = 1;
                    dm[l] = (float)(1.0 - c.damp_rate * sc2 * sc2);
                }
            }
            dmp = V2(dm[0], dm[1]);
        }
        bool bad = false;
#pragma unroll
        for (int f = 0; f < 12; f++) {
            // kicks with dt and dt/2 as fp32 pairs: the increment is formed first and
            // added in one rounding (lo*a folded into w first would be lost below
            // half an ulp and run the kick with fp32(dt))
            const V2 ha = fma2(hdt, acc[f], hdt_lo * acc[f]);
            V2 v = FIRST ? w[f] : w[f] + ha;
            if (DAMP && !FIRST) v = v * dmp;
            const V2 wn = (DAMP || FIRST) ? v + ha : w[f] + fma2(dt, acc[f], dt_lo * acc[f]);
            // compensated drift (hi, lo) += dt*w_{n+1}
            const V2 y = fma2(dt, wn, fma2(dt_lo, wn, bf16x2_to_v2(lo[f])));
            V2 xn, e;
            two_sum2(ctr[f], y, &xn, &e);
            *reinterpret_cast<uint32_t *>(io.loout + f * N3 + site) = v2_to_bf16x2(e);
            st_cs2(io.xout + f * N3 + site, xn);
            *reinterpret_cast<float2 *>(io.wout + f * N3 + site) = wn.v;
            if (SYNC && !FIRST) {
                st_cs2(io.sout + f * N3 + site, v);
                bad |= !isfinite(xn.v.x) || !isfinite(xn.v.y) || !isfinite(v.v.x) || !isfinite(v.v.y);
            }
        }
        if (GAUGED) {
            const V2 gad((float)c.gad), gad_lo((float)(c.gad - (double)(float)c.gad));
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const V2 hK = fma2(hdt, K[d], hdt_lo * K[d]);
                V2 E = FIRST ? w[FTH + d] : w[FTH + d] + hK;
                if (DAMP && !FIRST) E = E * dmp;
                const V2 Eh = (DAMP || FIRST) ? E + hK : w[FTH + d] + fma2(dt, K[d], dt_lo * K[d]);
                const V2 y = fma2(gad, Eh, fma2(gad_lo, Eh, S2(sc, NF + d, r0, cc)));
                V2 th, lnew;
                two_sum2(ctr[FTH + d], y, &th, &lnew);
                link_wrap_c(&th.v.x, &lnew.v.x);
                link_wrap_c(&th.v.y, &lnew.v.y);
                st_cs2(io.tloout + d * N3 + site, lnew);
                st_cs2(io.xout + (FTH + d) * N3 + site, th);
                *reinterpret_cast<float2 *>(io.wout + (FTH + d) * N3 + site) = Eh.v;
                if (SYNC && !FIRST) {
                    st_cs2(io.sout + (FTH + d) * N3 + site, E);
                    bad |= !isfinite(E.v.x) || !isfinite(E.v.y) || !isfinite(th.v.x) || !isfinite(th.v.y);
                }
            }
        }
        if (SYNC && bad) atomicOr(io.flag, 1);
#pragma unroll
        for (int f = 0; f < 12; f++) xm[f] = ctr[f];
    }
}

template <int TX, int TY, bool GAUGED, bool FIRST, bool SYNC, bool DAMP>
__global__ void __launch_bounds__(Step2Layout<TX, TY, GAUGED>::NT, Step2Layout<TX, TY, GAUGED>::MIN_BLOCKS)
step2_kernel(StepIO<F32C> io, StepConsts c, TileGrid tg) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for_each_piece(tg, c.N, [&](const Piece &pc) { step_item2<TX, TY, GAUGED, FIRST>(io, c, pc, SYNC, DAMP, smem_raw); });
}

// many FP32C requests of even N per launch (table semantics as step_multi_kernel)
template <int TX, int TY, bool GAUGED, bool DAMP>
__global__ void __launch_bounds__(Step2Layout<TX, TY, GAUGED>::NT, Step2Layout<TX, TY, GAUGED>::MIN_BLOCKS)
step2_multi_kernel(const ReqTable<F32C> *tab, int k) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nitems = tab->nitems, nreq = tab->nreq;
    const long long s = tab->step + k;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const ReqSlot<F32C> &q = tab->r[req_of_item(tab, nreq, item)];
        if (s < q.s0 || s >= q.s1) continue;       // uniform over the CTA
        const StepIO<F32C> io = q.io[(int)((s - q.s0) & 1)];
        const StepConsts c = q.c;
        const TileGrid tg = q.tg;
        step_item2<TX, TY, GAUGED, false>(io, c, piece_of_item(tg, item - q.item0, c.N), false, DAMP, smem_raw);
    }
}

}  // namespace scp
