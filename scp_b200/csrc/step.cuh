// step.cuh -- fused leapfrog step for the complex (v66) and gauged (v69)
// Cosserat Q-ball lattice, one launch per time step, in two precisions:
//   F64   all state and arithmetic in FP64 (the drop-in mode);
//   F32C  FP32 state and arithmetic; positions carried as a compensated pair
//         (hi: fp32, lo: bf16 for the matter fields, fp32 for the link
//         angles) so the drift accumulates without loss.
//         F32C evaluates Laplacians, currents and plaquette angles as sums of
//         neighbour differences, which removes the cancellation that FP32
//         would otherwise suffer against O(|f|) values.
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
// with the reference's arithmetic in the reference's order, so no
// acceleration array exists and each state word is read once and written
// once per step.  Links follow the same pattern with E and the wrapped drift
// th += -g*dx*dt*E.  The launch that starts a run (FIRST) reads v_0 instead
// of w and skips the stage-4 kick; a SYNC launch also stores v_{n+1} and
// E_{n+1} for diagnostics and snapshots.
//
// Data movement.  Persistent CTAs walk work items = (TX x TY) columns in
// (k, j) times segments of `seg` planes in i.  A CTA streams its column plane
// by plane through a 3-slot shared-memory ring (plane i, plane i+1, and plane
// i+2 in flight via cp.async), holding the x(i-1) centre values of its own
// sites in registers.  Every thread copies its own site; the halo rows and
// columns (periodic wrap) are spread over the CTA's threads so each thread
// issues the same copies with no per-field branches.  In gauged mode every
// thread evaluates the link cos/sin and plaquette sines it needs itself: its
// own site, the j-1 and k-1 neighbours (recomputed from the ring), and the
// i-1 values carried in registers from the previous plane -- more sines than
// sharing them through shared memory, but no extra barrier per plane and no
// shared array, which leaves room for more resident CTAs.
#pragma once
#include <cuda_bf16.h>

#include <type_traits>

#include "common.cuh"
#include "diag.cuh"
#include "trig.cuh"

namespace scp {

struct F64 {
    using T = double;
    static constexpr bool COMP = false;
};
struct F32C {
    using T = float;
    static constexpr bool COMP = true;
};

template <class P>
struct StepIO {
    using T = typename P::T;
    const T *xin;           // NF arrays of N^3: positions x_{n+1} (hi part in F32C)
    T *xout;                // NF arrays: x_{n+2}
    const uint16_t *loin;   // F32C: bf16 low parts of the 12 matter positions
    uint16_t *loout;
    const float *tloin;     // F32C gauged: low parts of the 3 link angles
    float *tloout;
    const T *win;           // NF arrays: w_n (or v_0, E_0 when FIRST)
    T *wout;                // NF arrays: w_{n+1} (may alias win)
    T *sout;                // NF arrays: v_{n+1}, E_{n+1} (SYNC only)
    int *flag;              // nonfinite flag (SYNC only)
    // FP64 SYNC launches of the single-grid kernel: when set, the launch also
    // sums the first diagnostics pass at (x_{n+1}, v_{n+1}) -- one partial of
    // DS_NSUM + DM_NMAX slots per CTA into dpart -- and stores the Gauss-law
    // charge density of every site into drho (gauged)
    double *dpart = nullptr;
    double *drho = nullptr;
};

template <class P, int TX, int TY, bool GAUGED>
struct StepLayout {
    using T = typename P::T;
    static constexpr int NF = GAUGED ? 15 : 12;
    static constexpr int NR = NF + ((P::COMP && GAUGED) ? 3 : 0);   // ring fields (+ link lo parts)
    static constexpr int PX = TX + 2, PY = TY + 2;
    static constexpr int PLANE = NR * PY * PX;            // elements per ring slot
    static constexpr int NT = TX * TY;
    static constexpr int NHALO = 2 * TX + 2 * TY + (GAUGED ? 2 : 0);
    static constexpr int HPT = (NHALO + NT - 1) / NT;      // halo sites per thread (max)
    static constexpr size_t smem_bytes = sizeof(T) * (size_t)(3 * PLANE);
};

__device__ __forceinline__ void cp_async_elem(double *s, const double *g) { cp_async8(s, g); }
__device__ __forceinline__ void cp_async_elem(float *s, const float *g) { cp_async4(s, g); }

__device__ __forceinline__ double ldg_t(const double *p) { return __ldg(p); }
__device__ __forceinline__ float ldg_t(const float *p) { return __ldg(p); }

__device__ __forceinline__ float bf16_to_f(uint16_t h) { return __uint_as_float((uint32_t)h << 16); }
__device__ __forceinline__ uint16_t f_to_bf16(float f) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}

// exact sum: s + e = a + b (Knuth two-sum)
__device__ __forceinline__ void two_sum(float a, float b, float *s, float *e) {
    const float t = a + b;
    const float bb = t - a;
    *e = (a - (t - bb)) + (b - bb);
    *s = t;
}

// link wrap into (-pi, pi] (reference: v - 2*pi*rint(v/(2*pi)), scp_sim.c:1647);
// |v| < 3 never wraps, so the division only runs for the rare large angles
__device__ __forceinline__ double link_wrap(double v) {
    if (fabs(v) < 3.0) return v;
    return wrap_angle(v);
}

// Plane staging of the classic ring: every thread copies its own site with
// cp.async, and the halo rows and columns (periodic wrap, two corners for
// the gauged plaquettes) are spread over the CTA's threads.  Slot layout
// [NR][PY][PX] of StepLayout; any grid size.
template <class P, int TX, int TY, bool GAUGED>
struct CpStage {
    using T = typename P::T;
    using LY = StepLayout<P, TX, TY, GAUGED>;
    static constexpr int NSLOT = 3;   // ring slots: planes i, i+1 resident, i+2 in flight
    static constexpr bool MOM = false;   // momenta read from global memory at the site
    __device__ __forceinline__ void issue_mom(int, int) {}
    __device__ __forceinline__ void wait_mom(int) {}
    __device__ __forceinline__ T mom(int, int) const { return T(0); }
    static constexpr int NF = LY::NF, NR = LY::NR, PX = LY::PX, PY = LY::PY, NT = LY::NT;
    T *xs;
    int N;
    long long N3;
    bool act;
    int oc, c_s;
    int h_s[LY::HPT], h_g[LY::HPT], h_nf[LY::HPT];

    __device__ __forceinline__ explicit CpStage(unsigned char *smem) : xs(reinterpret_cast<T *>(smem)) {}

    // per-item set-up: this thread's own site and its halo copies
    __device__ __forceinline__ void begin(const StepConsts &c, int k0, int j0, int nk, int nj) {
        N = c.N;
        N3 = c.N3;
        const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
        act = (tx < nk) && (ty < nj);
        oc = (j0 + ty) * N + k0 + tx;
        c_s = (ty + 1) * PX + tx + 1;
        const int jlo = wrapi(j0 - 1, N), jhi = wrapi(j0 + nj, N);
        const int klo = wrapi(k0 - 1, N), khi = wrapi(k0 + nk, N);
#pragma unroll
        for (int q = 0; q < LY::HPT; q++) {
            const int h = tid + q * NT;
            int r = 0, col = 0, gj = 0, gk = 0, nf = 0;
            if (h < nk) { r = 0; col = h + 1; gj = jlo; gk = k0 + h; nf = NF; }
            else if (h < 2 * nk) { r = nj + 1; col = h - nk + 1; gj = jhi; gk = k0 + h - nk; nf = NF; }
            else if (h < 2 * nk + nj) { r = h - 2 * nk + 1; col = 0; gj = j0 + h - 2 * nk; gk = klo; nf = NF; }
            else if (h < 2 * nk + 2 * nj) { r = h - 2 * nk - nj + 1; col = nk + 1; gj = j0 + h - 2 * nk - nj; gk = khi; nf = NF; }
            else if (GAUGED && h == 2 * nk + 2 * nj) { r = nj + 1; col = 0; gj = jhi; gk = klo; nf = 3; }
            else if (GAUGED && h == 2 * nk + 2 * nj + 1) { r = 0; col = nk + 1; gj = jlo; gk = khi; nf = 3; }
            h_s[q] = r * PX + col;
            h_g[q] = gj * N + gk;
            h_nf[q] = nf;
        }
    }

    __device__ __forceinline__ void issue(const StepIO<P> &io, int p, int slot) {
        const long long pb = (long long)wrapi(p, N) * N * N;
        T *sbase = xs + slot * LY::PLANE;
        const T *gbase = io.xin + pb;
        if (act) {
#pragma unroll
            for (int f = 0; f < NF; f++)
                cp_async_elem(sbase + f * PY * PX + c_s, gbase + f * N3 + oc);
            if constexpr (NR > NF) {
#pragma unroll
                for (int f = NF; f < NR; f++)
                    cp_async_elem(sbase + f * PY * PX + c_s, io.tloin + pb + (f - NF) * N3 + oc);
            }
        }
#pragma unroll
        for (int q = 0; q < LY::HPT; q++) {
            const int nf = h_nf[q];
            if (nf == 0) continue;
            const int f0 = (nf == NF) ? 0 : FTH;   // corners carry only the link angles
#pragma unroll
            for (int f = 0; f < NF; f++)
                if (f >= f0) cp_async_elem(sbase + f * PY * PX + h_s[q], gbase + f * N3 + h_g[q]);
            if constexpr (NR > NF) {
#pragma unroll
                for (int f = NF; f < NR; f++)
                    cp_async_elem(sbase + f * PY * PX + h_s[q], io.tloin + pb + (f - NF) * N3 + h_g[q]);
            }
        }
    }
    __device__ __forceinline__ void commit() { cp_async_commit(); }
    // this thread's copies have landed, all but the PENDING latest groups (a barrier follows)
    template <int PENDING>
    __device__ __forceinline__ void wait(int) { cp_async_wait<PENDING>(); }
    __device__ __forceinline__ bool failed() const { return false; }
    __device__ __forceinline__ T at(int slot, int f, int r, int col) const {
        return xs[((slot * NR + f) * PY + r) * PX + col];
    }
};

// One work item (a TX x TY column over one segment of planes) of one grid.
// sync and damp are uniform per call; the single-grid kernel passes them as
// constants, the multi-request kernel per request.  Stage stages the planes.
// Per-site gradient, coupling and plaquette terms of the gauged diagnostics
// (the energy's covariant gradients, eta (Phi . curl Theta), 1 - cos of the
// three plaquettes; compute_energy_complex_gauge, sfa/sim/scp_sim.c:1930-2036)
// for a synchronous FP64 launch that sums the first diagnostics pass: the
// covariant differences are formed again from the ring (planes i, i+1) and
// the thread's x(i-1).  Every input passes through an opaque copy first, so
// that none of this arithmetic can merge with the force's (which would change
// how the force's multiply-adds are fused): the launch advances the state bit
// for bit as one that sums nothing.
struct DiagGrad {
    double eg, etg, ec, bb;
};
struct Plane12 {
    double v[12];
};

__device__ __forceinline__ double opaque(double x) {
    asm("" : "+d"(x));
    return x;
}

template <int TX, int TY>
__device__ __forceinline__ DiagGrad diag_grad_gauged(const double *xs, int sc, int sp, int r, int col,
                                                     const Plane12 &xm_in, double c0m_in, double s0m_in,
                                                     double idx1_in) {
    constexpr int NR = 15, PX = TX + 2, PY = TY + 2;
    auto X = [&](int slot, int f, int rr, int cc) -> double {
        return opaque(xs[((slot * NR + f) * PY + rr) * PX + cc]);
    };
    Plane12 xm;
#pragma unroll
    for (int f = 0; f < 12; f++) xm.v[f] = opaque(xm_in.v[f]);
    const double c0m = opaque(c0m_in), s0m = opaque(s0m_in), idx1 = opaque(idx1_in);
    DiagGrad o{0.0, 0.0, 0.0, 0.0};
    double cr[3], ci[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        double cP, sP, cM, sM;
        sincos_bounded(X(sc, FTH + d, r, col), &sP, &cP);
        if (d == 0) { cM = c0m; sM = s0m; }
        else if (d == 1) sincos_bounded(X(sc, FTH + 1, r - 1, col), &sM, &cM);
        else sincos_bounded(X(sc, FTH + 2, r, col - 1), &sM, &cM);
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const int fre = q < 3 ? FU + q : FTU + q - 3, fim = q < 3 ? FV + q : FTV + q - 3;
            double up, vp, um, vm;
            if (d == 0) {
                up = X(sp, fre, r, col); vp = X(sp, fim, r, col);
                um = xm.v[fre]; vm = xm.v[fim];
            } else if (d == 1) {
                up = X(sc, fre, r + 1, col); vp = X(sc, fim, r + 1, col);
                um = X(sc, fre, r - 1, col); vm = X(sc, fim, r - 1, col);
            } else {
                up = X(sc, fre, r, col + 1); vp = X(sc, fim, r, col + 1);
                um = X(sc, fre, r, col - 1); vm = X(sc, fim, r, col - 1);
            }
            const double DR = ((cP * up - sP * vp) - (cM * um + sM * vm)) * idx1;
            const double DI = ((cP * vp + sP * up) - (cM * vm - sM * um)) * idx1;
            if (q < 3) o.eg += DR * DR + DI * DI;
            else o.etg += DR * DR + DI * DI;
            const int qa = q - 3;
            if (q >= 3 && qa != d) {   // curl of Theta: D_{a+1} Theta_{a+2} - D_{a+2} Theta_{a+1}
                if (qa == (d + 1) % 3) {
                    const int a = (d + 2) % 3;
                    if (d < (a + 2) % 3) { cr[a] = DR; ci[a] = DI; }
                    else { cr[a] = DR - cr[a]; ci[a] = DI - ci[a]; }
                } else {
                    const int a = (d + 1) % 3;
                    if (d < (a + 1) % 3) { cr[a] = DR; ci[a] = DI; }
                    else { cr[a] = cr[a] - DR; ci[a] = ci[a] - DI; }
                }
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++) o.ec += X(sc, FU + a, r, col) * cr[a] + X(sc, FV + a, r, col) * ci[a];
#pragma unroll
    for (int q = 0; q < 3; q++) {   // plaquette (q, q+1) at x, the next plane in slot sp
        const int a = q, b = (q + 1) % 3;
        const int sa = (a == 0) ? sp : sc, ra = r + (a == 1 ? 1 : 0), ca = col + (a == 2 ? 1 : 0);
        const int sb = (b == 0) ? sp : sc, rb = r + (b == 1 ? 1 : 0), cb = col + (b == 2 ? 1 : 0);
        double sn, cs;
        sincos_any(X(sc, FTH + a, r, col) + X(sa, FTH + b, ra, ca) - X(sb, FTH + a, rb, cb) - X(sc, FTH + b, r, col),
                   &sn, &cs);
        o.bb += 1.0 - cs;
    }
    return o;
}

// Per-thread sums and maxima of the first diagnostics pass kept in shared
// memory (slot q of thread t at q * NT + t), so that the synchronous launch
// that sums them keeps its registers for the force.
struct DiagSmem {
    double *base;
    int nt;
    struct Ref {
        double *p;
        int nt;
        __device__ __forceinline__ double &operator[](int q) const { return p[q * nt]; }
    };
    __device__ __forceinline__ Ref S() const { return Ref{base + threadIdx.x, nt}; }
    __device__ __forceinline__ Ref M() const { return Ref{base + DS_NSUM * nt + threadIdx.x, nt}; }
    static constexpr size_t bytes(int nt) { return sizeof(double) * kDiag1Q * (size_t)nt; }
};

// dsum (FP64 SYNC launches only): per-thread sums of the first diagnostics
// pass over this item's sites, the per-site terms of diag_ring.cuh / diag.cuh
// (compute_energy_complex[_gauge], compute_charges, sfa/sim/scp_sim.c:1823-2169)
// evaluated from the values the step holds; the Gauss-law slots are left to
// a pass that reads E of the neighbouring sites.
template <class P, int TX, int TY, bool GAUGED, bool FIRST, class Stage>
__device__ __forceinline__ void step_item(const StepIO<P> &io, const StepConsts &c, const Piece &pc,
                                          const bool SYNC, const bool DAMP, Stage &stg, const DiagSmem *dsum = nullptr) {
    const bool DG = !P::COMP && dsum != nullptr;
    using T = typename P::T;
    using LY = StepLayout<P, TX, TY, GAUGED>;
    constexpr int NF = LY::NF;
    constexpr int NR = LY::NR;
    auto XS = [&](int slot, int f, int r, int col) -> T { return stg.at(slot, f, r, col); };
    const int N = c.N;
    const long long N3 = c.N3;
    const int tid = threadIdx.x;
    const int tx = tid % TX, ty = tid / TX;
    const T dt = (T)c.dt, hdt = (T)c.hdt, idx1 = (T)c.idx1, idx2 = (T)c.idx2;
    const float dt_lo = (float)(c.dt - (double)(float)c.dt);
    const float hdt_lo = (float)(c.hdt - (double)(float)c.hdt);

    {
        const int k0 = pc.kt * TX, j0 = pc.jt * TY;
        const int i0 = pc.i0, i1 = pc.i1;
        const int k = k0 + tx, j = j0 + ty;
        const int nk = min(k0 + TX, N) - k0, nj = min(j0 + TY, N) - j0;   // valid extent of the tile
        const bool act = (tx < nk) && (ty < nj);
        const int oc = j * N + k;                                          // in-plane offset (act only)
        stg.begin(c, k0, j0, nk, nj);
        auto issue_plane = [&](int p, int slot) { stg.issue(io, p, slot); };

        // sine of the plaquette angle th_a(y) + th_b(y+a) - th_a(y+b) - th_b(y) of plane
        // (a,b) = (0,1) (1,2) (2,0) [q = 0, 1, 2] at ring position (r, col) of slot sc,
        // the next plane in slot sp (compute_forces_complex_gauge pass B, scp_sim.c:1090-1109)
        auto plaq_sin = [&](int q, int sc, int sp, int r, int col) -> T {
            const int a = q, b = (q + 1) % 3;
            // th_b(y+a): the next plane for a = 0, else the neighbour row (a = 1) or column (a = 2)
            const int sa = (a == 0) ? sp : sc, ra = r + (a == 1 ? 1 : 0), ca = col + (a == 2 ? 1 : 0);
            const int sb = (b == 0) ? sp : sc, rb = r + (b == 1 ? 1 : 0), cb = col + (b == 2 ? 1 : 0);
            const T tay = XS(sc, FTH + a, r, col), tby = XS(sc, FTH + b, r, col);
            const T tbya = XS(sa, FTH + b, ra, ca), tayb = XS(sb, FTH + a, rb, cb);
            if constexpr (NR > NF) {   // FP32C: hi differences plus lo differences
                const T hi = (tay - tayb) + (tbya - tby);
                const T lo = (XS(sc, NF + a, r, col) - XS(sb, NF + a, rb, cb)) +
                             (XS(sa, NF + b, ra, ca) - XS(sc, NF + b, r, col));
                return sin_bounded(hi + lo);
            } else {
                return sin_bounded(tay + tbya - tayb - tby);
            }
        };

        __syncthreads();   // previous item finished reading the ring
        issue_plane(i0 - 1, 0);
        issue_plane(i0, 1);
        stg.commit();
        stg.template wait<0>(0);
        stg.template wait<0>(1);
        __syncthreads();
        T xm[12];          // x(i-1) at this thread's site, matter fields
#pragma unroll
        for (int f = 0; f < 12; f++) xm[f] = act ? XS(0, f, ty + 1, tx + 1) : T(0);
        // link 0 and the (0,1), (2,0) plaquettes at x - i (carried from plane to plane)
        T c0m = T(1), s0m = T(0), P0m = T(0), P2m = T(0);
        if (GAUGED && act) {
            sincos_bounded(XS(0, FTH + 0, ty + 1, tx + 1), &s0m, &c0m);
            P0m = plaq_sin(0, 0, 1, ty + 1, tx + 1);
            P2m = plaq_sin(2, 0, 1, ty + 1, tx + 1);
        }
        // planes i0+1 .. i0+NS-2 (NS ring slots: NS-2 planes ahead in flight)
        constexpr int NS = Stage::NSLOT;
#pragma unroll
        for (int q = 1; q <= NS - 2; q++)
            if (i0 + q <= i1) issue_plane(i0 + q, q + 1);
        if constexpr (Stage::MOM) stg.issue_mom(i0, 0);   // momenta of the first plane
        stg.commit();

        for (int i = i0; i < i1; i++) {
            // plane p sits in slot (p - i0 + 1) mod NS; plane i + NS - 1 reuses the slot of i - 1
            const int sc = (i - i0 + 1) % NS, sp = (i - i0 + 2) % NS, sn = (i - i0) % NS;
            stg.template wait<NS - 3>(sp);   // the copies of planes beyond i+1 may stay in flight
            if constexpr (Stage::MOM) stg.wait_mom((i - i0) & 1);
            __syncthreads();
            if (i + NS - 1 <= i1) issue_plane(i + NS - 1, sn);
            if constexpr (Stage::MOM) {   // momenta of the next plane, into the slot plane i-1 used
                if (i + 1 < i1) stg.issue_mom(i + 1, (i + 1 - i0) & 1);
            }
            stg.commit();
            const long long site = (long long)i * N * N + oc;
            if (c.prefetch && act && i + 1 < i1) {
#pragma unroll
                for (int f = 0; f < NF; f++) prefetch_line_l2(io.win + f * N3 + site + (long long)N * N);
            }
            T w[NF];
            uint16_t lo[P::COMP ? 12 : 1];
            if (act) {
                if constexpr (Stage::MOM) {
#pragma unroll
                    for (int f = 0; f < NF; f++) w[f] = stg.mom((i - i0) & 1, f);
                } else {
#pragma unroll
                    for (int f = 0; f < NF; f++) w[f] = ldg_t(io.win + f * N3 + site);
                }
                if constexpr (P::COMP) {
#pragma unroll
                    for (int f = 0; f < 12; f++) lo[f] = __ldg(io.loin + f * N3 + site);
                }
            }
            if (!act) continue;
            // diagnostics: gradient, coupling and plaquette terms, formed before the
            // force while few of its values are live (link 0 at x - i is still the carry)
            DiagGrad gr{0.0, 0.0, 0.0, 0.0};
            if constexpr (!P::COMP && GAUGED && std::is_same<Stage, CpStage<P, TX, TY, GAUGED>>::value) {
                if (DG) {
                    Plane12 xp;
#pragma unroll
                    for (int f = 0; f < 12; f++) xp.v[f] = (double)xm[f];
                    gr = diag_grad_gauged<TX, TY>(stg.xs, sc, sp, ty + 1, tx + 1, xp, (double)c0m, (double)s0m,
                                                  c.idx1);
                }
            }

            T acc[12];
            T K[3] = {T(0), T(0), T(0)};
            T ctr[NF];
#pragma unroll
            for (int f = 0; f < NF; f++) ctr[f] = XS(sc, f, ty + 1, tx + 1);
            // potential pieces (scp_sim.c:946-958)
            const T s0 = ctr[FU + 0] * ctr[FU + 0] + ctr[FV + 0] * ctr[FV + 0];
            const T s1 = ctr[FU + 1] * ctr[FU + 1] + ctr[FV + 1] * ctr[FV + 1];
            const T s2 = ctr[FU + 2] * ctr[FU + 2] + ctr[FV + 2] * ctr[FV + 2];
            const T sp3 = s0 * s1 * s2;
            const T den = T(1) + (T)c.kappa * sp3;
            const T Vp = T(0.5) * (T)c.mu / (den * den);
            const T rest[3] = {s1 * s2, s0 * s2, s0 * s1};
            const T m2 = (T)c.m2, mt2 = (T)c.mtheta2, eta = (T)c.eta;

            if (!GAUGED) {
                // compute_forces_complex, scp_sim.c:931-994
                auto nb = [&](int f, int which) -> T {   // 0 ip 1 im 2 jp 3 jm 4 kp 5 km
                    switch (which) {
                        case 0: return XS(sp, f, ty + 1, tx + 1);
                        case 1: return xm[f];
                        case 2: return XS(sc, f, ty + 2, tx + 1);
                        case 3: return XS(sc, f, ty, tx + 1);
                        case 4: return XS(sc, f, ty + 1, tx + 2);
                        default: return XS(sc, f, ty + 1, tx);
                    }
                };
                auto lap = [&](int f) -> T {
                    if constexpr (P::COMP) {   // neighbour differences: no cancellation against 6*centre
                        const T x0 = ctr[f];
                        return ((nb(f, 0) - x0) + (nb(f, 1) - x0) + (nb(f, 2) - x0) + (nb(f, 3) - x0) +
                                (nb(f, 4) - x0) + (nb(f, 5) - x0)) * idx2;
                    } else {
                        return (nb(f, 0) + nb(f, 1) + nb(f, 2) + nb(f, 3) + nb(f, 4) + nb(f, 5) - T(6) * ctr[f]) * idx2;
                    }
                };
                auto curl = [&](int g0, int a) -> T {
                    if (a == 0) return (nb(g0 + 2, 2) - nb(g0 + 2, 3) - nb(g0 + 1, 4) + nb(g0 + 1, 5)) * idx1;
                    if (a == 1) return (nb(g0 + 0, 4) - nb(g0 + 0, 5) - nb(g0 + 2, 0) + nb(g0 + 2, 1)) * idx1;
                    return (nb(g0 + 1, 0) - nb(g0 + 1, 1) - nb(g0 + 0, 2) + nb(g0 + 0, 3)) * idx1;
                };
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    T x = ctr[FU + a];
                    acc[FU + a] = lap(FU + a) - m2 * x - T(2) * Vp * x * rest[a] + eta * curl(FTU, a);
                    x = ctr[FV + a];
                    acc[FV + a] = lap(FV + a) - m2 * x - T(2) * Vp * x * rest[a] + eta * curl(FTV, a);
                    x = ctr[FTU + a];
                    acc[FTU + a] = lap(FTU + a) - mt2 * x + eta * curl(FU, a);
                    x = ctr[FTV + a];
                    acc[FTV + a] = lap(FTV + a) - mt2 * x + eta * curl(FV, a);
                }
                if constexpr (!P::COMP) {
                    if (DG) {   // gradient energies and the Cosserat coupling energy
                        double eg = 0.0, etg = 0.0;
#pragma unroll
                        for (int d = 0; d < 3; d++) {
#pragma unroll
                            for (int q = 0; q < 6; q++) {
                                const int fre = q < 3 ? FU + q : FTU + q - 3, fim = q < 3 ? FV + q : FTV + q - 3;
                                // rounded products of their own (the step's fused ones stay as they are)
                                const double DR = __dmul_rn(nb(fre, 2 * d) - nb(fre, 2 * d + 1), idx1);
                                const double DI = __dmul_rn(nb(fim, 2 * d) - nb(fim, 2 * d + 1), idx1);
                                const double e2 = __fma_rn(DR, DR, __dmul_rn(DI, DI));
                                if (q < 3) eg += e2;
                                else etg += e2;
                            }
                        }
                        const auto S = dsum->S();
                        S[DS_EG] += 0.5 * eg * c.dV;
                        S[DS_ETG] += 0.5 * etg * c.dV;
#pragma unroll
                        for (int a = 0; a < 3; a++)
                            S[DS_EC] -= c.eta * (ctr[FU + a] * curl(FTU, a) + ctr[FV + a] * curl(FTV, a)) * c.dV;
                    }
                }
            } else {
                // compute_forces_complex_gauge pass C, scp_sim.c:1112-1262
                // complex fields q=0..2 Phi_a, q=3..5 Theta_a
                const T fu[6] = {ctr[FU], ctr[FU + 1], ctr[FU + 2], ctr[FTU], ctr[FTU + 1], ctr[FTU + 2]};
                const T fv[6] = {ctr[FV], ctr[FV + 1], ctr[FV + 2], ctr[FTV], ctr[FTV + 1], ctr[FTV + 2]};
                T lapU[6], lapV[6];
                // covariant curls, built as the directions come in: component a is
                // D[d = a+1][field a+2] - D[d = a+2][field a+1] (indices mod 3) of the
                // central differences D = (transported(x+d) - transported(x-d))/(2dx);
                // one subtraction either way round, as the reference forms it
                T crT[3], ciT[3], crP[3], ciP[3];
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    // link d at x (pass A, scp_sim.c:1072-1079) and at x - d
                    T cP, sP, cM, sM;
                    sincos_bounded(ctr[FTH + d], &sP, &cP);
                    if (d == 0) { cM = c0m; sM = s0m; c0m = cP; s0m = sP; }
                    else if (d == 1) sincos_bounded(XS(sc, FTH + 1, ty, tx + 1), &sM, &cM);
                    else sincos_bounded(XS(sc, FTH + 2, ty + 1, tx), &sM, &cM);
                    T TRpP[3], TIpP[3];   // forward transports of Phi
                    T tup[3], tvp[3];     // raw Theta at x+d (current and seagull)
#pragma unroll
                    for (int q = 0; q < 6; q++) {
                        const int fre = q < 3 ? FU + q : FTU + q - 3;
                        const int fim = q < 3 ? FV + q : FTV + q - 3;
                        T up, vp, um, vm;
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
                        const T TRp = cP * up - sP * vp, TIp = cP * vp + sP * up;
                        const T TRm = cM * um + sM * vm, TIm = cM * vm - sM * um;
                        if constexpr (P::COMP) {   // accumulate (transported - centre) differences
                            const T cu = fu[q], cv = fv[q];
                            if (d == 0) { lapU[q] = (TRp - cu) + (TRm - cu); lapV[q] = (TIp - cv) + (TIm - cv); }
                            else { lapU[q] = lapU[q] + (TRp - cu) + (TRm - cu); lapV[q] = lapV[q] + (TIp - cv) + (TIm - cv); }
                        } else {
                            if (d == 0) { lapU[q] = TRp + TRm; lapV[q] = TIp + TIm; }
                            else { lapU[q] = lapU[q] + TRp + TRm; lapV[q] = lapV[q] + TIp + TIm; }
                        }
                        const int qa = q < 3 ? q : q - 3;
                        if (qa != d) {
                            const T DR = (TRp - TRm) * idx1, DI = (TIp - TIm) * idx1;
                            T *cr = q < 3 ? crP : crT, *ci = q < 3 ? ciP : ciT;
                            if (qa == (d + 1) % 3) {            // plus term of a = d + 2
                                const int a = (d + 2) % 3;
                                if (d < (a + 2) % 3) { cr[a] = DR; ci[a] = DI; }
                                else { cr[a] = DR - cr[a]; ci[a] = DI - ci[a]; }
                            } else {                            // minus term of a = d + 1
                                const int a = (d + 1) % 3;
                                if (d < (a + 1) % 3) { cr[a] = DR; ci[a] = DI; }
                                else { cr[a] = cr[a] - DR; ci[a] = ci[a] - DI; }
                            }
                        }
                        if (q < 3) { TRpP[q] = TRp; TIpP[q] = TIp; }
                        else { tup[q - 3] = up; tvp[q - 3] = vp; }
                    }
                    // lattice current J (scp_sim.c:1232-1249); the Theta transports are
                    // recomputed from the cached raw neighbours to keep the live set small
                    T Jg = T(0);
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        const T TIt = cP * tvp[a] + sP * tup[a];
                        const T TRt = cP * tup[a] - sP * tvp[a];
                        if constexpr (P::COMP) {
                            // u*TI - v*TR = u*(TI - v) - v*(TR - u): differences of neighbouring
                            // values instead of a difference of two O(|f|^2) products
                            Jg += fu[a] * (TIpP[a] - fv[a]) - fv[a] * (TRpP[a] - fu[a]);
                            Jg += fu[3 + a] * (TIt - fv[3 + a]) - fv[3 + a] * (TRt - fu[3 + a]);
                        } else {
                            Jg += fu[a] * TIpP[a] - fv[a] * TRpP[a];
                            Jg += fu[3 + a] * TIt - fv[3 + a] * TRt;
                        }
                    }
                    const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
                    const T WpR1 = cP * fu[d2] + sP * fv[d2], WpI1 = cP * fv[d2] - sP * fu[d2];
                    const T WpR2 = cP * fu[d1] + sP * fv[d1], WpI2 = cP * fv[d1] - sP * fu[d1];
                    const T T12 = (fu[3 + d1] * TIpP[d2] - fv[3 + d1] * TRpP[d2])
                                + (tup[d1] * WpI1 - tvp[d1] * WpR1);
                    const T T21 = (fu[3 + d2] * TIpP[d1] - fv[3 + d2] * TRpP[d1])
                                + (tup[d2] * WpI2 - tvp[d2] * WpR2);
                    K[d] = (T)c.inva * Jg - T(0.5) * eta * (T12 - T21);   // Jlat; staple added below
                }
                // staples (scp_sim.c:1214-1220)
                const T P0 = plaq_sin(0, sc, sp, ty + 1, tx + 1), P1 = plaq_sin(1, sc, sp, ty + 1, tx + 1);
                const T P2 = plaq_sin(2, sc, sp, ty + 1, tx + 1);
                const T P0jm = plaq_sin(0, sc, sp, ty, tx + 1), P1jm = plaq_sin(1, sc, sp, ty, tx + 1);
                const T P1km = plaq_sin(1, sc, sp, ty + 1, tx), P2km = plaq_sin(2, sc, sp, ty + 1, tx);
                const T st0 = (P0 - P0jm) - (P2 - P2km);
                const T st1 = -(P0 - P0m) + (P1 - P1km);
                const T st2 = (P2 - P2m) - (P1 - P1jm);
                P0m = P0; P2m = P2;   // x - i of the next plane
                const T stp = (T)c.stp, gg = (T)c.g;
                K[0] = stp * st0 + gg * K[0];
                K[1] = stp * st1 + gg * K[1];
                K[2] = stp * st2 + gg * K[2];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const T c6 = P::COMP ? T(0) : T(6);   // FP32C accumulated differences already
                    const T lUP = (lapU[a] - c6 * fu[a]) * idx2;
                    const T lVP = (lapV[a] - c6 * fv[a]) * idx2;
                    const T lUT = (lapU[3 + a] - c6 * fu[3 + a]) * idx2;
                    const T lVT = (lapV[3 + a] - c6 * fv[3 + a]) * idx2;
                    acc[FU + a] = lUP - m2 * fu[a] - T(2) * Vp * fu[a] * rest[a] + eta * crT[a];
                    acc[FV + a] = lVP - m2 * fv[a] - T(2) * Vp * fv[a] * rest[a] + eta * ciT[a];
                    acc[FTU + a] = lUT - mt2 * fu[3 + a] + eta * crP[a];
                    acc[FTV + a] = lVT - mt2 * fv[3 + a] + eta * ciP[a];
                }
            }

            // kicks, damping, drift (scp_sim.c:1591-1715, fused)
            T dmp = T(1);
            if (DAMP && !FIRST) {
                const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
                const double r = sqrt(x * x + y * y + z * z);
                const double Rd = c.L - c.damp_width;
                if (r > Rd) {
                    double sc2 = (r - Rd) / c.damp_width;
                    if (sc2 > 1) sc2 = 1;
                    dmp = (T)(1.0 - c.damp_rate * sc2 * sc2);
                }
            }
            bool bad = false;
            double vv[NF];   // diagnostics: v_{n+1}, E_{n+1}
#pragma unroll
            for (int f = 0; f < 12; f++) {
                T v, wn, xn;
                if constexpr (P::COMP) {
                    // kicks with dt and dt/2 as fp32 pairs: the increment h*a is formed
                    // first (hi*a + lo*a), then added to the momentum in one rounding --
                    // folding lo*a into the momentum first would lose it below half an
                    // ulp and run the kick with fp32(dt), a systematic energy drift
                    const float ha = fmaf(hdt, acc[f], hdt_lo * acc[f]);
                    v = FIRST ? w[f] : w[f] + ha;
                    if (DAMP && !FIRST) v *= dmp;
                    if (DAMP || FIRST) wn = v + ha;
                    else wn = w[f] + fmaf((float)c.dt, acc[f], dt_lo * acc[f]);   // w_n + dt*a, no damping
                    // compensated drift (hi, lo) += dt*w_{n+1}
                    const float y = fmaf((float)c.dt, wn, fmaf(dt_lo, wn, bf16_to_f(lo[f])));
                    float e;
                    two_sum(ctr[f], y, &xn, &e);
                    io.loout[f * N3 + site] = f_to_bf16(e);
                } else {
                    v = FIRST ? w[f] : w[f] + hdt * acc[f];
                    if (DAMP && !FIRST) v *= dmp;
                    wn = v + hdt * acc[f];
                    xn = ctr[f] + dt * wn;
                    vv[f] = v;
                }
                st_cs(io.xout + f * N3 + site, xn);
                io.wout[f * N3 + site] = wn;
                if (SYNC && !FIRST) {
                    st_cs(io.sout + f * N3 + site, v);
                    bad |= !isfinite(xn) || !isfinite(v);
                }
            }
            if (GAUGED) {
                const T gad = (T)c.gad;
#pragma unroll
                for (int d = 0; d < 3; d++) {
                    T E, Eh, th;
                    if constexpr (P::COMP) {
                        const float hK = fmaf(hdt, K[d], hdt_lo * K[d]);
                        E = FIRST ? w[FTH + d] : w[FTH + d] + hK;
                        if (DAMP && !FIRST) E *= dmp;
                        if (DAMP || FIRST) Eh = E + hK;
                        else Eh = w[FTH + d] + fmaf((float)c.dt, K[d], dt_lo * K[d]);
                        const float gad_lo = (float)(c.gad - (double)(float)c.gad);
                        const float y = fmaf(gad, Eh, fmaf(gad_lo, Eh, XS(sc, NR - 3 + d, ty + 1, tx + 1)));
                        float lnew;
                        two_sum(ctr[FTH + d], y, &th, &lnew);
                        if (fabsf(th) > 3.0f) {   // wrap by 2 pi, carried as an fp32 pair
                            const float kq = rintf(th * 0.159154943091895336f);
                            float t1, e1;
                            two_sum(th, -kq * 6.28318548202514648f, &t1, &e1);   // 2 pi (fp32) times |kq| <= 1
                            lnew = lnew + e1 + kq * 1.74845553e-7f;              // 2 pi = 6.2831855f - 1.748e-7
                            two_sum(t1, lnew, &th, &lnew);
                        }
                        io.tloout[d * N3 + site] = lnew;
                    } else {
                        E = FIRST ? w[FTH + d] : w[FTH + d] + hdt * K[d];
                        if (DAMP && !FIRST) E *= dmp;
                        Eh = E + hdt * K[d];
                        th = link_wrap(ctr[FTH + d] + gad * Eh);
                        vv[FTH + d] = E;
                    }
                    st_cs(io.xout + (FTH + d) * N3 + site, th);
                    io.wout[(FTH + d) * N3 + site] = Eh;
                    if (SYNC && !FIRST) {
                        st_cs(io.sout + (FTH + d) * N3 + site, E);
                        bad |= !isfinite(E) || !isfinite(th);
                    }
                }
            }
            if (SYNC && bad) atomicOr(io.flag, 1);
            if constexpr (!P::COMP) {
                if (DG) {   // energies, charges, core and centroid moments at (x_{n+1}, v_{n+1})
                    // squares of the positions by rounded products of their own, so
                    // that they do not merge with the force's (whose fused
                    // multiply-adds would then change): the step's arithmetic is the
                    // same with and without these sums
                    const auto S = dsum->S();
                    const auto M = dsum->M();
                    const double dV = c.dV;
                    double s2[3];
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        const double u = ctr[FU + a], w0 = ctr[FV + a], tu = ctr[FTU + a], tv = ctr[FTV + a];
                        s2[a] = __fma_rn(u, u, __dmul_rn(w0, w0));
                        const double pu = vv[FU + a], pv = vv[FV + a], ptu = vv[FTU + a], ptv = vv[FTV + a];
                        S[DS_EPK] += 0.5 * (pu * pu + pv * pv) * dV;
                        S[DS_ETK] += 0.5 * (ptu * ptu + ptv * ptv) * dV;
                        S[DS_EM] += 0.5 * c.m2 * s2[a] * dV;
                        S[DS_ETM] += 0.5 * c.mtheta2 * __fma_rn(tu, tu, __dmul_rn(tv, tv)) * dV;
                        M[DM_PM] = fmax(M[DM_PM], sqrt(s2[a]));
                    }
                    const double s3 = s2[0] * s2[1] * s2[2];
                    S[DS_EP] += (c.mu / 2.0) * s3 / (1.0 + c.kappa * s3) * dV;
                    M[DM_PMAX] = fmax(M[DM_PMAX], sqrt(s3));
                    S[DS_PINT] += sqrt(s3) * dV;
#pragma unroll
                    for (int a = 0; a < 3; a++)
                        S[DS_TRS] += __fma_rn(ctr[FTU + a], ctr[FTU + a], __dmul_rn(ctr[FTV + a], ctr[FTV + a]));
                    const double x = -c.L + i * c.dx, y = -c.L + j * c.dx, z = -c.L + k * c.dx;
                    double rho2 = 0.0, qp = 0.0, qt = 0.0, sprod = 1.0;
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        const double qa = ctr[FU + a] * vv[FV + a] - ctr[FV + a] * vv[FU + a];
                        qp += qa;
                        S[DS_QP0 + a] += qa;
                        qt += ctr[FTU + a] * vv[FTV + a] - ctr[FTV + a] * vv[FTU + a];
                        const double s2a = s2[a];
                        rho2 += s2a;
                        sprod *= s2a;
                    }
                    S[DS_QP] += qp;
                    S[DS_QT] += qt;
                    if (x * x + y * y + z * z <= c.R2) S[DS_QC] += qp + qt;
                    M[DM_SMAX] = fmax(M[DM_SMAX], sprod);
                    S[DS_M0] += rho2;
                    S[DS_CX] += x * rho2;
                    S[DS_CY] += y * rho2;
                    S[DS_CZ] += z * rho2;
                    if constexpr (GAUGED && std::is_same<Stage, CpStage<P, TX, TY, GAUGED>>::value) {
                        // gradient, coupling and plaquette energies; Gauss charge density; E_em
                        S[DS_EG] += 0.5 * gr.eg * dV;
                        S[DS_ETG] += 0.5 * gr.etg * dV;
                        S[DS_EC] -= c.eta * gr.ec * dV;
                        const double bbE = gr.bb;
                        double rho = 0.0;
#pragma unroll
                        for (int a = 0; a < 3; a++)
                            rho += ctr[FU + a] * vv[FV + a] - ctr[FV + a] * vv[FU + a] +
                                   ctr[FTU + a] * vv[FTV + a] - ctr[FTV + a] * vv[FTU + a];
                        io.drho[site] = rho;
                        const double E0 = vv[FTH], E1 = vv[FTH + 1], E2 = vv[FTH + 2];
                        double ee = 0.5 * (E0 * E0 + E1 * E1 + E2 * E2);
                        ee += c.bpre * bbE;
                        S[DS_EEM] += ee * dV;
                    }
                }
            }
#pragma unroll
            for (int f = 0; f < 12; f++) xm[f] = ctr[f];
        }
    }
}

// Single grid: persistent CTAs over the grid's work items.
// resident CTAs per SM the register allocation is sized for
// (FP64 at 3 CTAs of 128 threads would spill the gauged force; FP32C fits)
template <class P, int TX, int TY, bool GAUGED>
struct MinBlocks {
    static constexpr int value = (TX * TY > 128) ? 1 : (P::COMP ? 3 : 2);
};

template <class P, int TX, int TY, bool GAUGED, bool FIRST, bool SYNC, bool DAMP>
__global__ void __launch_bounds__(TX * TY, (MinBlocks<P, TX, TY, GAUGED>::value))
step_kernel(StepIO<P> io, StepConsts c, TileGrid tg) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CpStage<P, TX, TY, GAUGED> stg(smem_raw);
    if constexpr (SYNC && !FIRST && !P::COMP) {
        if (io.dpart) {   // uniform: this launch also sums the first diagnostics pass
            using LY = StepLayout<P, TX, TY, GAUGED>;
            const DiagSmem dsm{reinterpret_cast<double *>(smem_raw + LY::smem_bytes), TX * TY};
#pragma unroll
            for (int q = 0; q < kDiag1Q; q++) dsm.base[q * TX * TY + threadIdx.x] = 0.0;
            for_each_piece(tg, c.N, [&](const Piece &pc) {
                step_item<P, TX, TY, GAUGED, FIRST>(io, c, pc, SYNC, DAMP, stg, &dsm);
            });
            __syncthreads();   // the ring is free: its first 7.4 KB serve as the fold's scratch
            DiagSums acc;
#pragma unroll
            for (int q = 0; q < DS_NSUM; q++) acc.S[q] = dsm.S()[q];
#pragma unroll
            for (int q = 0; q < DM_NMAX; q++) acc.M[q] = dsm.M()[q];
            block_fold<DS_NSUM, DM_NMAX>(acc.S, acc.M, reinterpret_cast<double *>(smem_raw), io.dpart);
            return;
        }
    }
    for_each_piece(tg, c.N, [&](const Piece &pc) { step_item<P, TX, TY, GAUGED, FIRST>(io, c, pc, SYNC, DAMP, stg); });
}

// ---------------------------------------------------------------- many grids per launch
//
// The serving loop advances every admitted request by one step per launch.
// Requests live in a device-resident table; request r is active for global
// steps s0 <= s < s1 and its buffers swap roles by the parity of s - s0.
// Because all of that is derived from the step counter in the table, the
// launches can be captured once in a CUDA graph and replayed while requests
// come and go: the host only rewrites the table between replays.  These
// launches never store the synchronous momenta: a request's final step (the
// one that does) runs through the single-grid kernel when it retires.  All
// requests of one launch share the damping mode (a template parameter).

constexpr int kMaxReq = 256;

template <class P>
struct ReqSlot {
    StepIO<P> io[2];      // io[p]: the step taken at parity p
    StepConsts c;
    TileGrid tg;
    int item0;            // first global work item of this request
    int pad;
    long long s0, s1;     // active global steps [s0, s1)
};

template <class P>
struct ReqTable {
    int nreq;
    int nitems;
    long long step;       // global step of launch k = 0 of the current replay
    ReqSlot<P> r[kMaxReq];
};

// last request of the table whose first item is <= item
template <class P>
__device__ __forceinline__ int req_of_item(const ReqTable<P> *tab, int nreq, int item) {
    int lo = 0, hi = nreq - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tab->r[mid].item0 <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <class P, int TX, int TY, bool GAUGED, bool DAMP>
__global__ void __launch_bounds__(TX * TY, (MinBlocks<P, TX, TY, GAUGED>::value))
step_multi_kernel(const ReqTable<P> *tab, int k) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nitems = tab->nitems, nreq = tab->nreq;
    const long long s = tab->step + k;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const ReqSlot<P> &q = tab->r[req_of_item(tab, nreq, item)];
        if (s < q.s0 || s >= q.s1) continue;       // uniform over the CTA
        // the request's arguments in registers: the table is global memory the
        // stores of the step could alias, so reading it in place reloads it
        const StepIO<P> io = q.io[(int)((s - q.s0) & 1)];
        const StepConsts c = q.c;
        const TileGrid tg = q.tg;
        CpStage<P, TX, TY, GAUGED> stg(smem_raw);
        step_item<P, TX, TY, GAUGED, false>(io, c, piece_of_item(tg, item - q.item0, c.N), false, DAMP, stg);
    }
}

}  // namespace scp
