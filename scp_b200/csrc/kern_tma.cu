// kern_tma.cu -- FP64 fused step kernels with TMA plane staging (tma.cuh).
#include "launch.cuh"
#include "tma.cuh"

namespace scp {
namespace {

template <int TX, int TY>
TmaStepFn pick_tma(bool g, bool f, bool s, bool d) {
    SCP_PICK16(step_tma_kernel, TX, TY);
}

template <int TX, int TY>
CpmStepFn pick_cpm(bool g, bool f, bool s, bool d) {
    SCP_PICK16(step_cpm_kernel, TX, TY);
}

}  // namespace

TmaStepFn step_tma_fn(int shape, bool g, bool f, bool s, bool d, size_t *smem) {
    if (shape == 2) {
        *smem = g ? TmaLayout<32, 8, true>::smem_bytes : TmaLayout<32, 8, false>::smem_bytes;
        return pick_tma<32, 8>(g, f, s, d);
    }
    *smem = g ? TmaLayout<32, 4, true>::smem_bytes : TmaLayout<32, 4, false>::smem_bytes;
    return pick_tma<32, 4>(g, f, s, d);
}

CpmStepFn step_cpm_fn(int shape, bool g, bool f, bool s, bool d, size_t *smem) {
    if (shape == 2) {
        *smem = g ? CpMomStage<32, 8, true>::smem_bytes : CpMomStage<32, 8, false>::smem_bytes;
        return pick_cpm<32, 8>(g, f, s, d);
    }
    *smem = g ? CpMomStage<32, 4, true>::smem_bytes : CpMomStage<32, 4, false>::smem_bytes;
    return pick_cpm<32, 4>(g, f, s, d);
}

}  // namespace scp
