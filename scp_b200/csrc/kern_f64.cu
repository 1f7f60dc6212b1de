// kern_f64.cu -- FP64 step kernels (single grid and multi-request).
#include "kern_one.cuh"

namespace scp {
StepFnT<F64> step_fn_f64(int shape, bool g, bool f, bool s, bool d, size_t *smem) {
    return select_one<F64>(shape, g, f, s, d, smem);
}
MultiFn<F64> multi_fn_f64(int shape, bool g, bool d, size_t *smem) {
    return select_multi<F64>(shape, g, d, smem);
}
}  // namespace scp
