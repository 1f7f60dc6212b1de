// kern_duo.cu -- gauged FP64 step kernels with two threads per site (step_duo.cuh).
#include "launch.cuh"
#include "step_duo.cuh"

namespace scp {
namespace {

template <int TX, int TY>
StepFnT<F64> pick_duo(bool f, bool s, bool d) {
    if (f) {
        if (s) return d ? step_duo_kernel<TX, TY, true, true, true> : step_duo_kernel<TX, TY, true, true, false>;
        return d ? step_duo_kernel<TX, TY, true, false, true> : step_duo_kernel<TX, TY, true, false, false>;
    }
    if (s) return d ? step_duo_kernel<TX, TY, false, true, true> : step_duo_kernel<TX, TY, false, true, false>;
    return d ? step_duo_kernel<TX, TY, false, false, true> : step_duo_kernel<TX, TY, false, false, false>;
}

}  // namespace

StepFnT<F64> step_duo_fn(bool f, bool s, bool d, size_t *smem) {
    *smem = DuoLayout<32, 4>::smem_bytes;
    return pick_duo<32, 4>(f, s, d);
}

}  // namespace scp
