// spectral.cuh -- direct solve of the periodic 7-point Poisson problem
//     -lap(chi) = b,   chi zero-mean,
// used as the starting point of the start-up Gauss projection's conjugate
// gradients (init_gauss_project, sfa/sim/scp_sim.c:2284-2400).  The discrete
// Laplacian on the periodic lattice is diagonal in the discrete Fourier basis
// with eigenvalues
//     -lambda(k) = -(4/dx^2) * sum_d sin^2(pi k_d / N),
// so chi_hat = b_hat / lambda for k != 0 and chi_hat(0) = 0.  This inverts the
// same operator the CG iterates on (not the continuum k^2), so the CG started
// from this chi finds its residual at round-off and stops after few or no
// iterations, with the reference's stopping rule unchanged.
//
// The 3-D transform is five passes of batched 1-D transforms over lines of
// the lattice, each line held in shared memory by one CTA together with
// B - 1 neighbouring lines (adjacent in k, or in j for the k lines) so that
// every global access is a run of B consecutive doubles:
//   pass 0  k lines   forward, real input b            -> (re, im)
//   pass 1  j lines   forward                          in place
//   pass 2  i lines   forward, divide by lambda*N^3, inverse   in place
//   pass 3  j lines   inverse                          in place
//   pass 4  k lines   inverse, real part                -> chi
// Power-of-two N uses radix-2 butterflies (decimation in time on bit-reversed
// input for forward transforms, decimation in frequency with bit-reversed
// output for inverse ones, so no permutation pass is needed); other N up to
// kDftMaxN use a direct O(N^2) transform per line.  Twiddle factors come from
// CUDA's sincospi.
#pragma once
#include "common.cuh"

namespace scp {

constexpr int kFftLines = 16;      // lines per CTA (16 doubles = one 128-byte run)
constexpr int kFftThreads = 256;
constexpr int kFftMaxN = 512;      // radix-2 path
constexpr int kDftMaxN = 192;      // direct path (N not a power of two)

__host__ __device__ constexpr bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

inline bool spectral_supported(int N) {
    return (is_pow2(N) && N >= 8 && N <= kFftMaxN) || (!is_pow2(N) && N >= 4 && N <= kDftMaxN);
}

// shared-memory bytes of one pass: re and im of B lines (row pitch N + 1,
// which keeps the B-strided accesses free of bank conflicts), a second set
// for the out-of-place direct transform, twiddles (cos, sin of 2 pi t / N)
// and the per-axis eigenvalue table
inline size_t spectral_smem_bytes(int N) {
    const size_t rows = (size_t)kFftLines * (N + 1);
    const size_t sets = is_pow2(N) ? 1 : 2;
    return sizeof(double) * (2 * rows * sets + 2 * (size_t)N + N);
}

inline int spectral_ctas(int N) { return N * ((N + kFftLines - 1) / kFftLines); }

struct FftLineMap {
    long long base;    // offset of line 0, position 0
    long long ms;      // stride between positions of a line
    long long ls;      // stride between the CTA's lines
    int a, b0, nl;     // plane index, first line, lines present (the last CTA of a plane may hold fewer)
};

// lines of pass `axis` (0: k, 1: j, 2: i) handled by CTA `cta`
__device__ __forceinline__ FftLineMap fft_lines(int axis, int N, int cta) {
    const long long NN = (long long)N * N;
    const int per = (N + kFftLines - 1) / kFftLines;     // CTAs per plane of lines
    const int a = cta / per, b0 = (cta % per) * kFftLines;
    FftLineMap m;
    m.a = a;
    m.b0 = b0;
    m.nl = min(kFftLines, N - b0);
    if (axis == 0) { m.base = (long long)a * NN + (long long)b0 * N; m.ms = 1; m.ls = N; }       // (i, j0..) rows
    else if (axis == 1) { m.base = (long long)a * NN + b0; m.ms = N; m.ls = 1; }                // (i, k0..)
    else { m.base = (long long)a * N + b0; m.ms = NN; m.ls = 1; }                               // (j, k0..)
    return m;
}

__device__ __forceinline__ int bit_reverse(int v, int bits) { return (int)(__brev((unsigned)v) >> (32 - bits)); }

// radix-2 decimation in time over B lines in place; input bit-reversed,
// output natural.  sgn = -1 forward, +1 inverse.
__device__ __forceinline__ void fft_dit(double *re, double *im, int N, int pitch, const double *twc,
                                        const double *tws, double sgn) {
    const int half_n = N >> 1;
    for (int h = 1; h < N; h <<= 1) {
        const int tstep = N / (2 * h);
        for (int q = threadIdx.x; q < kFftLines * half_n; q += blockDim.x) {
            const int l = q / half_n, p = q - l * half_n;
            const int pos = p & (h - 1), i0 = ((p - pos) << 1) + pos, i1 = i0 + h;
            const int t = pos * tstep;
            const double c = twc[t], s = sgn * tws[t];
            double *R = re + l * pitch, *I = im + l * pitch;
            const double xr = R[i1], xi = I[i1];
            const double tr = c * xr - s * xi, ti = c * xi + s * xr;
            const double ar = R[i0], ai = I[i0];
            R[i0] = ar + tr; I[i0] = ai + ti;
            R[i1] = ar - tr; I[i1] = ai - ti;
        }
        __syncthreads();
    }
}

// radix-2 decimation in frequency in place; input natural, output bit-reversed
__device__ __forceinline__ void fft_dif(double *re, double *im, int N, int pitch, const double *twc,
                                        const double *tws, double sgn) {
    const int half_n = N >> 1;
    for (int h = half_n; h >= 1; h >>= 1) {
        const int tstep = N / (2 * h);
        for (int q = threadIdx.x; q < kFftLines * half_n; q += blockDim.x) {
            const int l = q / half_n, p = q - l * half_n;
            const int pos = p & (h - 1), i0 = ((p - pos) << 1) + pos, i1 = i0 + h;
            const int t = pos * tstep;
            const double c = twc[t], s = sgn * tws[t];
            double *R = re + l * pitch, *I = im + l * pitch;
            const double ar = R[i0], ai = I[i0], br = R[i1], bi = I[i1];
            R[i0] = ar + br; I[i0] = ai + bi;
            const double dr = ar - br, di = ai - bi;
            R[i1] = c * dr - s * di; I[i1] = c * di + s * dr;
        }
        __syncthreads();
    }
}

// direct transform out[m] = sum_n in[n] exp(sgn 2 pi i m n / N), out of place
__device__ __forceinline__ void dft_direct(const double *re, const double *im, double *ore, double *oim, int N,
                                           int pitch, const double *twc, const double *tws, double sgn) {
    for (int q = threadIdx.x; q < kFftLines * N; q += blockDim.x) {
        const int l = q / N, m = q - l * N;
        const double *R = re + l * pitch, *I = im + l * pitch;
        double sr = 0.0, si = 0.0;
        int t = 0;
        for (int n = 0; n < N; n++) {
            const double c = twc[t], s = sgn * tws[t];
            sr += c * R[n] - s * I[n];
            si += c * I[n] + s * R[n];
            t += m;
            if (t >= N) t -= N;
        }
        ore[l * pitch + m] = sr;
        oim[l * pitch + m] = si;
    }
    __syncthreads();
}

// One pass (see the file comment).  in_re/in_im and out_re/out_im may alias
// (in-place passes); in_im == nullptr reads a real input.
template <bool POW2>
__global__ void __launch_bounds__(kFftThreads) spectral_pass_kernel(int pass, int N, double inv_dx2,
                                                                     const double *in_re, const double *in_im,
                                                                     double *out_re, double *out_im) {
    extern __shared__ __align__(16) double fsm[];
    const int pitch = N + 1;
    const int rows = kFftLines * pitch;
    double *re = fsm, *im = fsm + rows;
    double *re2 = im + rows, *im2 = re2 + (POW2 ? 0 : rows);
    double *twc = POW2 ? re2 : im2 + rows;
    double *tws = twc + N, *lam = tws + N;
    const int nt = POW2 ? N / 2 : N;      // twiddles needed
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)t / (double)N, &s, &c);
        twc[t] = c;
        tws[t] = s;
    }
    const int axis = (pass == 0 || pass == 4) ? 0 : (pass == 2 ? 2 : 1);
    if (pass == 2)
        for (int t = threadIdx.x; t < N; t += blockDim.x) {
            const double s = sinpi((double)t / (double)N);
            lam[t] = 4.0 * inv_dx2 * s * s;
        }
    const FftLineMap mp = fft_lines(axis, N, blockIdx.x);
    const bool forward_first = pass <= 2;
    int bits = 0;
    if (POW2) while ((1 << bits) < N) bits++;

    // load: runs of B consecutive doubles along ls = 1, whole rows along ms = 1
    for (int e = threadIdx.x; e < kFftLines * N; e += blockDim.x) {
        int l, m;
        if (mp.ls == 1) { l = e % kFftLines; m = e / kFftLines; }
        else { m = e % N; l = e / N; }
        const int d = (POW2 && forward_first) ? bit_reverse(m, bits) : m;
        double vr = 0.0, vi = 0.0;
        if (l < mp.nl) {
            const long long g = mp.base + (long long)l * mp.ls + (long long)m * mp.ms;
            vr = in_re[g];
            vi = in_im ? in_im[g] : 0.0;
        }
        re[l * pitch + d] = vr;
        im[l * pitch + d] = vi;
    }
    __syncthreads();

    double *fre = re, *fim = im;   // where the result of the transforms lands
    if (forward_first) {
        if (POW2) fft_dit(re, im, N, pitch, twc, tws, -1.0);
        else { dft_direct(re, im, re2, im2, N, pitch, twc, tws, -1.0); fre = re2; fim = im2; }
    }
    if (pass == 2) {
        // line (j = a, k = b0 + l) after the k and j passes holds wavenumbers (kj, kk);
        // position m is ki; divide by lambda and the 1/N^3 of the unnormalised pair
        const int kj = mp.a, kk0 = mp.b0;
        const double n3inv = 1.0 / ((double)N * (double)N * (double)N);
        for (int e = threadIdx.x; e < mp.nl * N; e += blockDim.x) {
            const int l = e / N, m = e - l * N;
            const double lm = lam[m] + lam[kj] + lam[kk0 + l];
            const double f = (lm > 0.0) ? n3inv / lm : 0.0;   // zero mode: chi has zero mean
            fre[l * pitch + m] *= f;
            fim[l * pitch + m] *= f;
        }
        __syncthreads();
    }
    if (pass >= 2) {
        if (POW2) fft_dif(fre, fim, N, pitch, twc, tws, +1.0);
        else {
            double *ore = (fre == re) ? re2 : re, *oim = (fre == re) ? im2 : im;
            dft_direct(fre, fim, ore, oim, N, pitch, twc, tws, +1.0);
            fre = ore; fim = oim;
        }
    }
    // store (bit-reversed positions after a DIF)
    for (int e = threadIdx.x; e < kFftLines * N; e += blockDim.x) {
        int l, m;
        if (mp.ls == 1) { l = e % kFftLines; m = e / kFftLines; }
        else { m = e % N; l = e / N; }
        if (l >= mp.nl) continue;
        const long long g = mp.base + (long long)l * mp.ls + (long long)m * mp.ms;
        const int s = (POW2 && pass >= 2) ? bit_reverse(m, bits) : m;
        out_re[g] = fre[l * pitch + s];
        if (out_im) out_im[g] = fim[l * pitch + s];
    }
}

}  // namespace scp
