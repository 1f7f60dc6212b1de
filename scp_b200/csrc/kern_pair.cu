// kern_pair.cu -- two-site packed FP32-compensated step kernels (even N).
#include "launch.cuh"

namespace scp {
namespace {

template <int TX, int TY>
StepFnT<F32C> pick_pair(bool g, bool f, bool s, bool d) {
    SCP_PICK16(step2_kernel, TX, TY);
}

template <int TX, int TY>
size_t smem_pair(bool g) {
    return g ? Step2Layout<TX, TY, true>::smem_bytes : Step2Layout<TX, TY, false>::smem_bytes;
}

}  // namespace

StepFnT<F32C> step2_fn(int shape, bool g, bool f, bool s, bool d, size_t *smem) {
    switch (shape) {
        case 2: *smem = smem_pair<32, 8>(g); return pick_pair<32, 8>(g, f, s, d);
        case 3: *smem = smem_pair<16, 8>(g); return pick_pair<16, 8>(g, f, s, d);
        case 4: *smem = smem_pair<64, 2>(g); return pick_pair<64, 2>(g, f, s, d);
        default: *smem = smem_pair<32, 4>(g); return pick_pair<32, 4>(g, f, s, d);
    }
}

template <int TX, int TY>
static MultiFn<F32C> pick_multi2(bool g, bool d) {
    SCP_PICK4(step2_multi_kernel, TX, TY);
}

MultiFn<F32C> multi2_fn(int shape, bool g, bool d, size_t *smem) {
    switch (shape) {
        case 2: *smem = smem_pair<32, 8>(g); return pick_multi2<32, 8>(g, d);
        case 3: *smem = smem_pair<16, 8>(g); return pick_multi2<16, 8>(g, d);
        case 4: *smem = smem_pair<64, 2>(g); return pick_multi2<64, 2>(g, d);
        default: *smem = smem_pair<32, 4>(g); return pick_multi2<32, 4>(g, d);
    }
}

}  // namespace scp
