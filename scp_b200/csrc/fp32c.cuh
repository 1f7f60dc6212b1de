// fp32c.cuh -- FP32-compensated precision mode (placeholder until the mode's
// kernels land; every entry point reports SCP_EUNSUPPORTED).
#pragma once
#include "common.cuh"

namespace scp {

struct Fp32cState {
    long long bytes = 0;
    double state_bytes_per_site = 0.0;
};

inline cudaError_t fp32c_occupancy(int, int, int, int *occ) { *occ = 0; return cudaSuccess; }
inline int fp32c_init(Fp32cState *, const StepConsts &, int, const double *, const double *, int, int,
                      const TileGrid &, int, bool, int *, cudaStream_t) { return -7; }
inline int fp32c_step(Fp32cState *, bool, cudaStream_t) { return -7; }
inline int fp32c_expand(Fp32cState *, double *, double *, cudaStream_t) { return -7; }
inline void fp32c_free(Fp32cState *) {}
inline const char *fp32c_last_error() { return "FP32C mode not built"; }

}  // namespace scp
