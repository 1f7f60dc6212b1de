// kern_ext.cu -- instantiations and launchers of the extension steppers'
// ring kernels (Higgs condensate / second gauge, three fabrics).
#include <stdlib.h>

#include "diag_ring.cuh"
#include "ext_launch.cuh"
#include "fabrics.cuh"
#include "higgs_u1.cuh"
#include "real6.cuh"

namespace scp {

namespace {

// L2 prefetch of the next plane's momenta in the ring kernels: on unless
// SCP_RING_PREFETCH=0 in the environment (read once)
int ring_prefetch() {
    static const int on = [] {
        const char *e = getenv("SCP_RING_PREFETCH");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return on;
}

// Tile of a ring model: 128 threads, so that two CTAs share an SM and one
// CTA's plane barrier overlaps the other's work; 32 x 4 while the 4-slot ring
// of NR fields fits twice in shared memory, 16 x 8 (narrower halo rows) for
// the widest rings.
template <class M>
struct TileOf {
    static constexpr int TX = (M::NR <= 17) ? 32 : 16;
    static constexpr int TY = (M::NR <= 17) ? 4 : 8;
    static constexpr int NT = TX * TY;
};

template <class M>
int ring_plan(int N, int nsm, ExtPlan *p) {
    constexpr int TX = TileOf<M>::TX, TY = TileOf<M>::TY;
    using S = RingShape<M::NR, TX, TY>;
    auto fn = ring_kernel<M, TX, TY>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem_bytes) != cudaSuccess)
        return -1;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, TX * TY, S::smem_bytes) != cudaSuccess || occ < 1)
        return -1;
    plan_ring_tiles(N, TX, TY, nsm * occ, p);
    p->smem = S::smem_bytes;
    return 0;
}

template <bool H, bool G>
cudaError_t hu_launch(const ExtPlan &p, const HuConsts &c, const HuIO &io, cudaStream_t st) {
    using M = HiggsU1<H, G>;
    typename M::Args a;
    const long long n3 = c.N3;
    for (int f = 0; f < M::NR; f++) a.src.f[f] = io.x + f * n3;
    a.src.prefetch = ring_prefetch();
    a.N = c.N;
    a.c = c;
    a.win = io.win;
    a.wout = io.wout;
    a.xout = io.xout;
    a.sout = io.sout;
    a.flag = io.flag;
    a.first = io.first;
    a.sync = io.sync;
    a.damp = io.damp;
    ring_kernel<M, TileOf<M>::TX, TileOf<M>::TY><<<p.grid, TileOf<M>::NT, p.smem, st>>>(a, p.tg);
    return cudaGetLastError();
}

}  // namespace

int hu_plan(bool higgs, bool g2, int N, int nsm, ExtPlan *plan) {
    if (higgs && g2) return ring_plan<HiggsU1<true, true>>(N, nsm, plan);
    if (higgs) return ring_plan<HiggsU1<true, false>>(N, nsm, plan);
    return ring_plan<HiggsU1<false, true>>(N, nsm, plan);
}

cudaError_t hu_step(bool higgs, bool g2, const ExtPlan &plan, const HuConsts &c, const HuIO &io, cudaStream_t st) {
    if (higgs && g2) return hu_launch<true, true>(plan, c, io, st);
    if (higgs) return hu_launch<true, false>(plan, c, io, st);
    return hu_launch<false, true>(plan, c, io, st);
}

int fabric_plan(int N, int nsm, ExtPlan *fabric, ExtPlan *second, ExtPlan *link) {
    if (ring_plan<FabricPass<false>>(N, nsm, fabric)) return -1;
    if (ring_plan<FabricPass<true>>(N, nsm, second)) return -1;
    return ring_plan<LinkPass>(N, nsm, link);
}

namespace {
template <bool SECOND>
cudaError_t fabric_launch(const ExtPlan &p, const FabConsts &c, const FabIO &io, cudaStream_t st) {
    using M = FabricPass<SECOND>;
    typename M::Args a;
    const long long n3 = c.N3;
    for (int f = 0; f < 12; f++) a.src.f[f] = io.x + f * n3;
    for (int d = 0; d < 3; d++) a.src.f[M::TH + d] = io.th + d * n3;
    a.src.prefetch = ring_prefetch();
    a.N = c.N;
    a.c = c;
    a.qf = io.qf;
    a.gqf = io.gqf;
    a.qx = io.qx;
    a.gqx = io.gqx;
    a.win = io.win;
    a.wout = io.wout;
    a.xout = io.xout;
    a.sout = io.sout;
    a.kacc = io.kacc;
    a.flag = io.flag;
    a.first = io.first;
    a.sync = io.sync;
    a.damp = io.damp;
    a.accumulate = io.accumulate;
    ring_kernel<M, TileOf<M>::TX, TileOf<M>::TY><<<p.grid, TileOf<M>::NT, p.smem, st>>>(a, p.tg);
    return cudaGetLastError();
}
}  // namespace

cudaError_t fabric_step(const ExtPlan &plan, const FabConsts &c, const FabIO &io, cudaStream_t st) {
    return io.second ? fabric_launch<true>(plan, c, io, st) : fabric_launch<false>(plan, c, io, st);
}

cudaError_t link_step(const ExtPlan &p, const FabConsts &c, const LinkIO &io, cudaStream_t st) {
    LinkPass::Args a;
    const long long n3 = c.N3;
    for (int d = 0; d < 3; d++) a.src.f[d] = io.th + d * n3;
    a.src.prefetch = ring_prefetch();
    a.N = c.N;
    a.c = c;
    a.kacc = io.kacc;
    a.win = io.win;
    a.wout = io.wout;
    a.xout = io.thout;
    a.sout = io.sout;
    a.flag = io.flag;
    a.first = io.first;
    a.sync = io.sync;
    a.damp = io.damp;
    using T = TileOf<LinkPass>;
    ring_kernel<LinkPass, T::TX, T::TY><<<p.grid, T::NT, p.smem, st>>>(a, p.tg);
    return cudaGetLastError();
}

namespace {
template <bool G>
int diag_plan_t(int N, int nsm, ExtPlan *p) {
    using M = DiagRing<G>;
    constexpr int TX = TileOf<M>::TX, TY = TileOf<M>::TY;
    using S = RingShape<M::NR, TX, TY>;
    auto fn = diag_ring_kernel<G, TX, TY>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem_bytes) != cudaSuccess)
        return -1;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, TX * TY, S::smem_bytes) != cudaSuccess || occ < 1)
        return -1;
    plan_ring_tiles(N, TX, TY, nsm * occ, p);
    p->smem = S::smem_bytes;
    return 0;
}
template <bool G>
cudaError_t diag_launch_t(const ExtPlan &p, const DiagConsts &c, const DiagRingIO &io, double *part,
                          cudaStream_t st) {
    typename DiagRing<G>::Args a;
    for (int f = 0; f < 12; f++) a.src.f[f] = io.x[f];
    for (int d = 0; d < 3; d++) {   // without links: any valid arrays, never read
        a.src.f[DiagRing<G>::TH + d] = io.th ? io.th + d * c.N3 : io.x[d];
        a.src.f[DiagRing<G>::EF + d] = io.E ? io.E + d * c.N3 : io.x[3 + d];
    }
    a.N = c.N;
    a.c = c;
    a.mom = io.mom;
    using T = TileOf<DiagRing<G>>;
    diag_ring_kernel<G, T::TX, T::TY><<<p.grid, T::NT, p.smem, st>>>(a, p.tg, part);
    return cudaGetLastError();
}
}  // namespace

int diag_ring_plan(bool gauged, bool, int N, int nsm, ExtPlan *plan) {
    return gauged ? diag_plan_t<true>(N, nsm, plan) : diag_plan_t<false>(N, nsm, plan);
}

cudaError_t diag_ring_pass1(bool gauged, bool, const ExtPlan &plan, const DiagConsts &c, const DiagRingIO &io,
                            double *part, cudaStream_t st) {
    return gauged ? diag_launch_t<true>(plan, c, io, part, st) : diag_launch_t<false>(plan, c, io, part, st);
}

int r6_plan(bool aux, int N, int nsm, ExtPlan *aux_plan, ExtPlan *step_plan) {
    if (aux) {
        if (ring_plan<R6Aux>(N, nsm, aux_plan)) return -1;
        return ring_plan<R6Step<true>>(N, nsm, step_plan);
    }
    return ring_plan<R6Step<false>>(N, nsm, step_plan);
}

namespace {
template <bool AUX>
cudaError_t r6_launch(const ExtPlan &p, const R6Consts &c, const R6IO &io, cudaStream_t st) {
    using M = R6Step<AUX>;
    typename M::Args a;
    const long long n3 = c.N3;
    for (int f = 0; f < 6; f++) a.src.f[f] = io.x + f * n3;
    if (AUX)
        for (int f = 0; f < 6; f++) a.src.f[6 + f] = io.aux + f * n3;
    a.N = c.N;
    a.c = c;
    a.win = io.win;
    a.wout = io.wout;
    a.xout = io.xout;
    a.sout = io.sout;
    a.flag = io.flag;
    a.first = io.first;
    a.sync = io.sync;
    a.damp = io.damp;
    ring_kernel<M, TileOf<M>::TX, TileOf<M>::TY><<<p.grid, TileOf<M>::NT, p.smem, st>>>(a, p.tg);
    return cudaGetLastError();
}
}  // namespace

cudaError_t r6_step(const ExtPlan &aux_plan, const ExtPlan &step_plan, const R6Consts &c, const R6IO &io,
                    cudaStream_t st) {
    if (!io.aux) return r6_launch<false>(step_plan, c, io, st);
    R6Aux::Args a;
    for (int f = 0; f < 6; f++) a.src.f[f] = io.x + f * c.N3;
    a.N = c.N;
    a.c = c;
    a.aux = io.aux;
    using T = TileOf<R6Aux>;
    ring_kernel<R6Aux, T::TX, T::TY><<<aux_plan.grid, T::NT, aux_plan.smem, st>>>(a, aux_plan.tg);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return r6_launch<true>(step_plan, c, io, st);
}

}  // namespace scp
