// kern_one.cuh -- selectors of the one-site step kernels of one precision,
// included by kern_f64.cu / kern_f32c.cu with SCP_PREC set.
#pragma once
#include "launch.cuh"

namespace scp {
namespace {

template <class P, int TX, int TY>
StepFnT<P> pick_one(bool g, bool f, bool s, bool d) {
    SCP_PICK16(step_kernel, P, TX, TY);
}

template <class P, int TX, int TY>
size_t smem_one(bool g) {
    return g ? StepLayout<P, TX, TY, true>::smem_bytes : StepLayout<P, TX, TY, false>::smem_bytes;
}

// the synchronous FP64 launches also hold the diagnostics sums (DiagSmem)
template <class P, int TX, int TY>
size_t smem_variant(bool g, bool f, bool s) {
    return smem_one<P, TX, TY>(g) + ((s && !f && !P::COMP) ? DiagSmem::bytes(TX * TY) : 0);
}

template <class P>
StepFnT<P> select_one(int shape, bool g, bool f, bool s, bool d, size_t *smem) {
    switch (shape) {
        case 2: *smem = smem_variant<P, 32, 8>(g, f, s); return pick_one<P, 32, 8>(g, f, s, d);
        case 3: *smem = smem_variant<P, 16, 8>(g, f, s); return pick_one<P, 16, 8>(g, f, s, d);
        case 4: *smem = smem_variant<P, 64, 2>(g, f, s); return pick_one<P, 64, 2>(g, f, s, d);
        default: *smem = smem_variant<P, 32, 4>(g, f, s); return pick_one<P, 32, 4>(g, f, s, d);
    }
}

template <class P, int TX, int TY>
MultiFn<P> pick_multi(bool g, bool d) {
    SCP_PICK4(step_multi_kernel, P, TX, TY);
}

template <class P>
MultiFn<P> select_multi(int shape, bool g, bool d, size_t *smem) {
    switch (shape) {
        case 2: *smem = smem_one<P, 32, 8>(g); return pick_multi<P, 32, 8>(g, d);
        case 3: *smem = smem_one<P, 16, 8>(g); return pick_multi<P, 16, 8>(g, d);
        case 4: *smem = smem_one<P, 64, 2>(g); return pick_multi<P, 64, 2>(g, d);
        default: *smem = smem_one<P, 32, 4>(g); return pick_multi<P, 32, 4>(g, d);
    }
}

}  // namespace
}  // namespace scp
