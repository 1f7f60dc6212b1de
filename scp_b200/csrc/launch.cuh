// launch.cuh -- host-side selection of the compiled step kernels.
//
// The step kernels are instantiated in their own translation units
// (kern_f64.cu, kern_f32c.cu, kern_pair.cu) so they compile in parallel; this
// header declares the selectors that return a kernel's host stub and its
// dynamic shared-memory size for a tile shape and variant.
#pragma once
#include <cuda.h>
#include <stddef.h>

#include "step.cuh"
#include "step2.cuh"

namespace scp {

template <class P>
using StepFnT = void (*)(StepIO<P>, StepConsts, TileGrid);
template <class P>
using MultiFn = void (*)(const ReqTable<P> *, int);

struct TileShape { int tx, ty; };
// tile_variant 1..: fixed shapes; 0 picks the default for the mode
constexpr TileShape kShapes[] = {{32, 4}, {32, 4}, {32, 8}, {16, 8}, {64, 2}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

// one-site kernels: g gauged, f first step, s synchronous momenta, d damping
StepFnT<F64> step_fn_f64(int shape, bool g, bool f, bool s, bool d, size_t *smem);
StepFnT<F32C> step_fn_f32c(int shape, bool g, bool f, bool s, bool d, size_t *smem);
// multi-request kernels: g gauged, d damping
MultiFn<F64> multi_fn_f64(int shape, bool g, bool d, size_t *smem);
MultiFn<F32C> multi_fn_f32c(int shape, bool g, bool d, size_t *smem);
// two-site packed FP32C kernels (even N)
StepFnT<F32C> step2_fn(int shape, bool g, bool f, bool s, bool d, size_t *smem);
MultiFn<F32C> multi2_fn(int shape, bool g, bool d, size_t *smem);

// FP64 kernels with TMA plane staging (tma.cuh; shapes 1 and 2, full tiles only)
struct TmaMaps;
using TmaStepFn = void (*)(StepIO<F64>, StepConsts, TileGrid, const TmaMaps);
TmaStepFn step_tma_fn(int shape, bool g, bool f, bool s, bool d, size_t *smem);
// FP64 kernels with the cp.async position ring and TMA-staged momenta (tma.cuh)
using CpmStepFn = void (*)(StepIO<F64>, StepConsts, TileGrid, const CUtensorMap);
CpmStepFn step_cpm_fn(int shape, bool g, bool f, bool s, bool d, size_t *smem);

// gauged FP64 kernels with two threads per site (step_duo.cuh; tile 32 x 4)
StepFnT<F64> step_duo_fn(bool f, bool s, bool d, size_t *smem);

template <class P>
StepFnT<P> step_fn(int shape, bool g, bool f, bool s, bool d, size_t *smem);
template <>
inline StepFnT<F64> step_fn<F64>(int shape, bool g, bool f, bool s, bool d, size_t *smem) {
    return step_fn_f64(shape, g, f, s, d, smem);
}
template <>
inline StepFnT<F32C> step_fn<F32C>(int shape, bool g, bool f, bool s, bool d, size_t *smem) {
    return step_fn_f32c(shape, g, f, s, d, smem);
}
template <class P>
MultiFn<P> multi_fn(int shape, bool g, bool d, size_t *smem);
template <>
inline MultiFn<F64> multi_fn<F64>(int shape, bool g, bool d, size_t *smem) { return multi_fn_f64(shape, g, d, smem); }
template <>
inline MultiFn<F32C> multi_fn<F32C>(int shape, bool g, bool d, size_t *smem) { return multi_fn_f32c(shape, g, d, smem); }

#define SCP_PICK4(KERNEL, ...)                                                                     \
    do {                                                                                           \
        if (g) return d ? KERNEL<__VA_ARGS__, true, true> : KERNEL<__VA_ARGS__, true, false>;       \
        return d ? KERNEL<__VA_ARGS__, false, true> : KERNEL<__VA_ARGS__, false, false>;            \
    } while (0)

// Instantiation helpers for the kern_*.cu units.
#define SCP_PICK16(KERNEL, ...)                                                                        \
    do {                                                                                               \
        if (g) {                                                                                       \
            if (f) {                                                                                   \
                if (s) return d ? KERNEL<__VA_ARGS__, true, true, true, true>                           \
                                : KERNEL<__VA_ARGS__, true, true, true, false>;                         \
                return d ? KERNEL<__VA_ARGS__, true, true, false, true>                                 \
                         : KERNEL<__VA_ARGS__, true, true, false, false>;                               \
            }                                                                                          \
            if (s) return d ? KERNEL<__VA_ARGS__, true, false, true, true>                              \
                            : KERNEL<__VA_ARGS__, true, false, true, false>;                            \
            return d ? KERNEL<__VA_ARGS__, true, false, false, true> : KERNEL<__VA_ARGS__, true, false, false, false>; \
        }                                                                                              \
        if (f) {                                                                                       \
            if (s) return d ? KERNEL<__VA_ARGS__, false, true, true, true>                              \
                            : KERNEL<__VA_ARGS__, false, true, true, false>;                            \
            return d ? KERNEL<__VA_ARGS__, false, true, false, true> : KERNEL<__VA_ARGS__, false, true, false, false>; \
        }                                                                                              \
        if (s) return d ? KERNEL<__VA_ARGS__, false, false, true, true>                                 \
                        : KERNEL<__VA_ARGS__, false, false, true, false>;                               \
        return d ? KERNEL<__VA_ARGS__, false, false, false, true> : KERNEL<__VA_ARGS__, false, false, false, false>; \
    } while (0)

}  // namespace scp
