// kern_f32c.cu -- one-site FP32-compensated step kernels (odd N).
#include "kern_one.cuh"

namespace scp {
StepFnT<F32C> step_fn_f32c(int shape, bool g, bool f, bool s, bool d, size_t *smem) {
    return select_one<F32C>(shape, g, f, s, d, smem);
}
MultiFn<F32C> multi_fn_f32c(int shape, bool g, bool d, size_t *smem) {
    return select_multi<F32C>(shape, g, d, smem);
}
}  // namespace scp
