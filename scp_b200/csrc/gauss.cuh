// gauss.cuh -- start-up constraint handling of the gauged stepper, on device:
// the net-charge check (net_charge_check, sfa/sim/scp_sim.c:2264-2279) and the
// one-time Gauss projection (init_gauss_project, :2284-2400): conjugate
// gradients on -lap(chi) = G - mean(G) with the periodic 7-point Laplacian,
// chi kept zero-mean, then E_d += (chi(x+d) - chi(x))/dx and the frozen
// offset G_offset = mean(G).  The reference runs this on the host even in its
// CUDA build (scp_sim.cu:5151-5155); here every sweep is a kernel and all
// dot products use the deterministic reductions of reduce.cuh.
#pragma once
#include "reduce.cuh"

namespace scp {

struct GaussArgs {
    const double *X;   // positions (u v tu tv th), 15 arrays
    double *S;         // momenta (du dv dtu dtv E), 15 arrays; E updated in place
    int N;
    long long N3;
    double dx, g;
};

__device__ __forceinline__ double rho_site(const GaussArgs &a, long long idx) {
    double r = 0.0;
    for (int c = 0; c < 3; c++)
        r += a.X[(FU + c) * a.N3 + idx] * a.S[(FV + c) * a.N3 + idx]
           - a.X[(FV + c) * a.N3 + idx] * a.S[(FU + c) * a.N3 + idx]
           + a.X[(FTU + c) * a.N3 + idx] * a.S[(FTV + c) * a.N3 + idx]
           - a.X[(FTV + c) * a.N3 + idx] * a.S[(FTU + c) * a.N3 + idx];
    return r;
}

__device__ __forceinline__ double gauss_site(const GaussArgs &a, long long idx) {
    const int N = a.N;
    const long long NN = (long long)N * N;
    int i, j, k;
    site_ijk(idx, N, &i, &j, &k);
    const double *E0 = a.S + (FTH + 0) * a.N3, *E1 = a.S + (FTH + 1) * a.N3, *E2 = a.S + (FTH + 2) * a.N3;
    const long long im = (long long)wrapi(i - 1, N) * NN + (long long)j * N + k;
    const long long jm = (long long)i * NN + (long long)wrapi(j - 1, N) * N + k;
    const long long km = (long long)i * NN + (long long)j * N + wrapi(k - 1, N);
    const double divE = (E0[idx] - E0[im] + E1[idx] - E1[jm] + E2[idx] - E2[km]) / a.dx;
    return divE - a.g * rho_site(a, idx);
}

// sums of rho*dV and |rho|*dV
__global__ void __launch_bounds__(kRedThreads) net_charge_kernel(GaussArgs a, double dV, double *part) {
    __shared__ double scratch[2 * 32];
    double S[2] = {0.0, 0.0}, M[1] = {0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < a.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        const double r = rho_site(a, idx);
        S[0] += r * dV;
        S[1] += fabs(r) * dV;
    }
    block_fold<2, 0>(S, M, scratch, part);
}

// b = G(x); partial sum of b
__global__ void __launch_bounds__(kRedThreads) gauss_rhs_kernel(GaussArgs a, double *b, double *part) {
    __shared__ double scratch[32];
    double S[1] = {0.0}, M[1] = {0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < a.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        const double G = gauss_site(a, idx);
        b[idx] = G;
        S[0] += G;
    }
    block_fold<1, 0>(S, M, scratch, part);
}

// CG scalars kept on the device
enum : int { CG_GBAR = 0, CG_GMAX0, CG_RZ, CG_PAP, CG_ALPHA, CG_BETA, CG_XBAR, CG_RMAX, CG_RZ2, CG_TOL, CG_DONE,
             CG_IT, CG_N };

// The iteration loop runs on the device in batches: every launch returns at
// once when CG_DONE is set (residual below tolerance or iteration cap), so the
// host only checks after a batch and the iterations taken are exactly those
// of the reference's while (rmax > tol && it < itmax) loop.

// b -= gbar; r = p = b; chi = 0; partial sum r^2, max |b|
__global__ void __launch_bounds__(kRedThreads) cg_start_kernel(long long n3, double *b, double *r, double *p,
                                                               double *x, const double *cg, double *part) {
    __shared__ double scratch[2 * 32];
    double S[1] = {0.0}, M[1] = {0.0};
    const double gbar = cg[CG_GBAR];
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n3;
         idx += (long long)gridDim.x * blockDim.x) {
        const double v = b[idx] - gbar;
        b[idx] = v; r[idx] = v; p[idx] = v; x[idx] = 0.0;
        M[0] = fmax(M[0], fabs(v));
        S[0] += v * v;
    }
    block_fold<1, 1>(S, M, scratch, part);
}

// One CG iteration is two launches.  The last CTA to finish each launch folds
// the per-CTA partials (fold_partials_block, the same fixed-order fold as
// everywhere else) and updates the scalars, so no separate fold or scalar
// launches are needed; the arithmetic and its order are those of the
// reference loop (init_gauss_project, scp_sim.c:2330-2364).

// p_new = r + beta*p_old (the reference's direction update, applied here at
// the start of the next iteration), x -= xbar, Ap = -lap(p_new); p_new at the
// six neighbours is formed on the fly with the same expression, so it equals
// what their owners store.  The last CTA sets alpha = rz / (p.Ap).
__global__ void __launch_bounds__(kRedThreads) cg_dirapply_kernel(int N, long long n3, double idx2, const double *r,
                                                                  const double *pold, double *pnew, double *x,
                                                                  double *Ap, double *part, unsigned *count,
                                                                  double *fold, double *cg) {
    __shared__ double scratch[32];
    double S[1] = {0.0}, M[1] = {0.0};
    if (cg[CG_DONE] != 0.0) return;              // uniform: set by an earlier launch
    const double beta = cg[CG_BETA], xbar = cg[CG_XBAR];
    const long long NN = (long long)N * N;
    auto P = [&](long long y) { return fma(beta, pold[y], r[y]); };
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        const double pc = P(idx);
        const double lap = (P((long long)wrapi(i + 1, N) * NN + (long long)j * N + k)
                            + P((long long)wrapi(i - 1, N) * NN + (long long)j * N + k)
                            + P((long long)i * NN + (long long)wrapi(j + 1, N) * N + k)
                            + P((long long)i * NN + (long long)wrapi(j - 1, N) * N + k)
                            + P((long long)i * NN + (long long)j * N + wrapi(k + 1, N))
                            + P((long long)i * NN + (long long)j * N + wrapi(k - 1, N)) - 6.0 * pc) * idx2;
        pnew[idx] = pc;
        x[idx] -= xbar;
        const double ap = -lap;
        Ap[idx] = ap;
        S[0] += pc * ap;
    }
    block_fold<1, 0>(S, M, scratch, part);
    if (last_block_done(count)) {
        fold_partials_block<1, 0>(part, gridDim.x, fold);
        __syncthreads();
        if (threadIdx.x == 0) {
            cg[CG_PAP] = fold[0];
            cg[CG_ALPHA] = cg[CG_RZ] / fold[0];
        }
    }
}

// x += alpha p; r -= alpha Ap; the last CTA sets rz, xbar, beta, max|r|,
// counts the iteration and decides whether to go on.
__global__ void __launch_bounds__(kRedThreads) cg_update_kernel(long long n3, double *x, double *r, const double *p,
                                                                const double *Ap, double *part, unsigned *count,
                                                                double *fold, double *cg, double n3d, int itmax) {
    __shared__ double scratch[3 * 32];
    double S[2] = {0.0, 0.0}, M[1] = {0.0};
    if (cg[CG_DONE] != 0.0) return;
    const double alpha = cg[CG_ALPHA];
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n3;
         idx += (long long)gridDim.x * blockDim.x) {
        const double xv = x[idx] + alpha * p[idx];
        const double rv = r[idx] - alpha * Ap[idx];
        x[idx] = xv; r[idx] = rv;
        S[0] += rv * rv;
        S[1] += xv;
        M[0] = fmax(M[0], fabs(rv));
    }
    block_fold<2, 1>(S, M, scratch, part);
    if (last_block_done(count)) {
        fold_partials_block<2, 1>(part, gridDim.x, fold);
        __syncthreads();
        if (threadIdx.x == 0) {
            cg[CG_RZ2] = fold[0];
            cg[CG_XBAR] = fold[1] / n3d;
            cg[CG_BETA] = fold[0] / cg[CG_RZ];
            cg[CG_RZ] = fold[0];
            cg[CG_RMAX] = fold[2];
            cg[CG_IT] += 1.0;
            if (!(cg[CG_RMAX] > cg[CG_TOL]) || cg[CG_IT] >= (double)itmax) cg[CG_DONE] = 1.0;
        }
    }
}

// Warm start from a given chi (the spectral solve, spectral.cuh): r = b - A chi
// = b + lap(chi) computed explicitly, p = r; partial sums r^2 and chi, max |r|.
// The CG then goes on from chi with the unchanged stopping rule.
__global__ void __launch_bounds__(kRedThreads) cg_warm_kernel(int N, long long n3, double idx2, const double *b,
                                                              const double *x, double *r, double *p, double *part) {
    __shared__ double scratch[3 * 32];
    double S[2] = {0.0, 0.0}, M[1] = {0.0};
    const long long NN = (long long)N * N;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        const double xc = x[idx];
        const double lap = (x[(long long)wrapi(i + 1, N) * NN + (long long)j * N + k]
                            + x[(long long)wrapi(i - 1, N) * NN + (long long)j * N + k]
                            + x[(long long)i * NN + (long long)wrapi(j + 1, N) * N + k]
                            + x[(long long)i * NN + (long long)wrapi(j - 1, N) * N + k]
                            + x[(long long)i * NN + (long long)j * N + wrapi(k + 1, N)]
                            + x[(long long)i * NN + (long long)j * N + wrapi(k - 1, N)] - 6.0 * xc) * idx2;
        const double rv = b[idx] + lap;
        r[idx] = rv;
        p[idx] = rv;
        S[0] += rv * rv;
        S[1] += xc;
        M[0] = fmax(M[0], fabs(rv));
    }
    block_fold<2, 1>(S, M, scratch, part);
}

// single-thread scalar bookkeeping of the start-up
__global__ void cg_scalar_kernel(int stage, double n3d, const double *fold, double *cg) {
    if (threadIdx.x | blockIdx.x) return;
    switch (stage) {
        case 0: cg[CG_GBAR] = fold[0] / n3d; break;                          // gbar
        case 1:
            cg[CG_RZ] = fold[0]; cg[CG_GMAX0] = fold[1]; cg[CG_RMAX] = fold[1];
            cg[CG_TOL] = 1e-13 * fmax(1.0, fold[1]);
            cg[CG_IT] = 0.0;
            cg[CG_BETA] = 0.0;     // first direction p = r
            cg[CG_XBAR] = 0.0;
            cg[CG_DONE] = (fold[1] > cg[CG_TOL]) ? 0.0 : 1.0;
            break;
        case 2:   // after cg_warm_kernel: the residual of the starting chi decides
            cg[CG_RZ] = fold[0];
            cg[CG_XBAR] = fold[1] / n3d;
            cg[CG_RMAX] = fold[2];
            cg[CG_BETA] = 0.0;
            cg[CG_IT] = 0.0;
            cg[CG_DONE] = (fold[2] > cg[CG_TOL]) ? 0.0 : 1.0;
            break;
    }
}

// E_d += (chi(x+d) - chi(x))/dx with chi = x - xbar: the reference's last
// iteration subtracts xbar in its direction step, which the next
// cg_dirapply_kernel would have done here
__global__ void gauss_correct_kernel(GaussArgs a, const double *x, const double *cg) {
    const int N = a.N;
    const long long NN = (long long)N * N;
    const double xbar = cg[CG_XBAR];
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < a.N3;
         idx += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        site_ijk(idx, N, &i, &j, &k);
        const double c0 = x[idx] - xbar;
        a.S[(FTH + 0) * a.N3 + idx] += ((x[(long long)wrapi(i + 1, N) * NN + (long long)j * N + k] - xbar) - c0) / a.dx;
        a.S[(FTH + 1) * a.N3 + idx] += ((x[(long long)i * NN + (long long)wrapi(j + 1, N) * N + k] - xbar) - c0) / a.dx;
        a.S[(FTH + 2) * a.N3 + idx] += ((x[(long long)i * NN + (long long)j * N + wrapi(k + 1, N)] - xbar) - c0) / a.dx;
    }
}

// partial sums of G (for G_offset)
__global__ void __launch_bounds__(kRedThreads) gauss_sum_kernel(GaussArgs a, double *part) {
    __shared__ double scratch[32];
    double S[1] = {0.0}, M[1] = {0.0};
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < a.N3;
         idx += (long long)gridDim.x * blockDim.x)
        S[0] += gauss_site(a, idx);
    block_fold<1, 0>(S, M, scratch, part);
}

}  // namespace scp
