// common.cuh -- shared device-side definitions of libscpgpu (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace scp {

// Packed field slots used by every device buffer.  Positions X: u0..2 v0..2
// tu0..2 tv0..2 th0..2; momenta W/S: du0..2 dv0..2 dtu0..2 dtv0..2 E0..2.
enum : int { FU = 0, FV = 3, FTU = 6, FTV = 9, FTH = 12 };

// Constants of one stepper instance, passed by value (kernel parameter bank).
struct StepConsts {
    int N;
    long long N3;
    double idx2, idx1, inva;      // 1/dx^2, 1/(2dx), 1/dx
    double m2, mtheta2, eta, mu, kappa;
    double dt, hdt, gad;          // gad = -g*dx*dt (link drift prefactor)
    double g, stp;                // stp = 1/(g dx^3) (staple prefactor)
    double L, dx, damp_width, damp_rate;
    int prefetch;                 // 1: prefetch the next plane's momenta into L2 at the top of a plane
    // diagnostics summed by synchronous FP64 launches: cell volume, core
    // radius^2 of Q_core, plaquette-energy prefactor 1/(g^2 dx^4)
    double dV, R2, bpre;
};

// Work decomposition of the persistent step kernels: the grid is cut into
// (TX x TY) columns in (k, j) and segments of seg planes along i.
struct TileGrid {
    int ntx, nty, nseg, seg;
    int nitems;
};

// A run of planes [i0, i1) of column (kt, jt).
struct Piece {
    int kt, jt, i0, i1;
};

// Work item -> piece.  Items enumerate the columns fastest and the segments
// last, so the CTAs of one wave start on the same plane and walk i in step.
__device__ __forceinline__ Piece piece_of_item(const TileGrid &tg, int item, int N) {
    Piece p;
    p.kt = item % tg.ntx;
    p.jt = (item / tg.ntx) % tg.nty;
    const int sg = item / (tg.ntx * tg.nty);
    p.i0 = sg * tg.seg;
    p.i1 = min(p.i0 + tg.seg, N);
    return p;
}

// Every piece of this CTA, in order (items blockIdx.x, + gridDim.x, ...).
template <class F>
__device__ __forceinline__ void for_each_piece(const TileGrid &tg, int N, F &&f) {
    for (int item = blockIdx.x; item < tg.nitems; item += gridDim.x) f(piece_of_item(tg, item, N));
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND) : "memory");
}

// Bring the line holding p into L2 ahead of its use (a hint: no register, no wait).
__device__ __forceinline__ void prefetch_line_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

// Streaming store (evict-first): outputs are not re-read by this launch.
__device__ __forceinline__ void st_cs(double *p, double v) { __stcs(p, v); }
__device__ __forceinline__ void st_cs(float *p, float v) { __stcs(p, v); }

// Link-angle wrap to (-pi, pi], the reference's v - 2*pi*rint(v/(2*pi))
// (sfa/sim/scp_sim.c:1647).
__device__ __forceinline__ double wrap_angle(double v) {
    const double twopi = 2.0 * 3.14159265358979323846;
    return v - twopi * rint(v / twopi);
}

__device__ __forceinline__ int wrapi(int x, int N) { return x < 0 ? x + N : (x >= N ? x - N : x); }

// (i, j, k) of site idx = (i*N + j)*N + k: 32-bit divisions while the index
// fits (N <= 1625), 64-bit beyond
__device__ __forceinline__ void site_ijk(long long idx, int N, int *i, int *j, int *k) {
    if (idx <= 0xFFFFFFFFll) {
        const unsigned u = (unsigned)idx, n = (unsigned)N, nn = n * n;
        const unsigned ii = u / nn, r = u - ii * nn, jj = r / n;
        *i = (int)ii;
        *j = (int)jj;
        *k = (int)(r - jj * n);
    } else {
        const long long NN = (long long)N * N;
        *i = (int)(idx / NN);
        *j = (int)((idx / N) % N);
        *k = (int)(idx % N);
    }
}

}  // namespace scp
