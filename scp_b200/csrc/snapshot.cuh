// snapshot.cuh -- device-side column packing and down-conversion for SFA
// snapshots (sfa_snap, sfa/sim/scp_sim.c:2646-2700; downcast kernels
// sfa/sim/scp_sim.cu:1734-1751).
#pragma once
#include "common.cuh"

namespace scp {

// Source slot of SFA column c (registration order, scp_sim.c:2862-2897):
// returns the packed field index and whether it lives in the momentum buffer.
__host__ __device__ inline void sfa_col_source(int c, int *field, int *momentum) {
    const int grp = c / 3, a = c % 3;
    static const int kField[10] = {FU, FTU, FU, FTU, FV, FTV, FV, FTV, FTH, FTH};
    static const int kMom[10] = {0, 0, 1, 1, 0, 0, 1, 1, 0, 1};
    *field = kField[grp] + a;
    *momentum = kMom[grp];
}

// IEEE half from a double the way the reference's f64_to_f16 does it
// (sfa/sim/scp_config.h:548-559): round to float, then truncate the mantissa,
// flush results below the half normal range to signed zero and send
// overflow (and NaN) to signed infinity.
__host__ __device__ inline uint16_t f64_to_f16_trunc(double v) {
    const float f = (float)v;
    uint32_t x;
#ifdef __CUDA_ARCH__
    x = __float_as_uint(f);
#else
    memcpy(&x, &f, 4);
#endif
    const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
    const int e = (int)((x >> 23) & 0xFFu) - 127 + 15;
    const uint16_t mant = (uint16_t)((x >> 13) & 0x3FFu);
    if (e <= 0) return sign;
    if (e >= 31) return (uint16_t)(sign | 0x7C00u);
    return (uint16_t)(sign | (e << 10) | mant);
}

__global__ void cast_f32_kernel(const double *src, float *dst, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}
__global__ void cast_f16_kernel(const double *src, uint16_t *dst, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = f64_to_f16_trunc(src[i]);
}

}  // namespace scp
