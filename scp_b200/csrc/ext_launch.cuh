// ext_launch.cuh -- host-side launchers of the extension steppers' ring
// kernels (higgs_u1.cuh, fabrics.cuh), instantiated in kern_ext.cu so they
// compile in their own nvcc process.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include "common.cuh"

namespace scp {

struct HuConsts;
struct FabConsts;
struct R6Consts;
struct DiagConsts;

// Launch geometry of one ring kernel: tile shape, work items, CTAs.
struct ExtPlan {
    int tx = 0, ty = 0;
    TileGrid tg{};
    int grid = 0;
    size_t smem = 0;
};

// Segment length along i that minimises waves x (planes + 2 halo planes) over
// `slots` resident CTAs, as the fused step plans its tiles.
inline void plan_ring_tiles(int N, int tx, int ty, int slots, ExtPlan *p) {
    TileGrid tg;
    tg.ntx = (N + tx - 1) / tx;
    tg.nty = (N + ty - 1) / ty;
    const int ntiles = tg.ntx * tg.nty;
    double best = 1e300;
    int best_seg = N;
    for (int s = 2; s <= N; s = (s < 16) ? s + 2 : s + s / 2) {
        const long long items = (long long)ntiles * ((N + s - 1) / s);
        const double cost = (double)((items + slots - 1) / slots) * (s + 2);
        if (cost < best - 1e-9) { best = cost; best_seg = s; }
    }
    const double whole = (double)((ntiles + slots - 1) / slots) * (N + 2);
    if (whole < best - 1e-9) best_seg = N;
    tg.seg = best_seg;
    tg.nseg = (N + best_seg - 1) / best_seg;
    tg.nitems = ntiles * tg.nseg;
    p->tx = tx;
    p->ty = ty;
    p->grid = tg.nitems < slots ? tg.nitems : slots;
    p->tg = tg;
}

// Higgs condensate and / or second gauge: positions and momenta are NR
// consecutive N^3 arrays (matter, th, [th2], [H]; matter, E, [E2], [dH/dt]).
struct HuIO {
    const double *x;      // x_{n+1}
    double *xout;         // x_{n+2}
    const double *win;    // w_n, or v_0 on the first launch
    double *wout, *sout;
    int *flag;
    int first, sync, damp;
};
int hu_plan(bool higgs, bool g2, int N, int nsm, ExtPlan *plan);
cudaError_t hu_step(bool higgs, bool g2, const ExtPlan &plan, const HuConsts &c, const HuIO &io, cudaStream_t st);

// One fabric's matter step, and the shared links' step.
struct FabIO {
    const double *x;      // the fabric's 12 matter positions x_{n+1}
    const double *th;     // the 3 link angles x_{n+1}
    double *xout;         // 12 matter positions x_{n+2}
    const double *win;    // 12 momenta
    double *wout, *sout;
    double *kacc;         // 3 arrays of accumulated currents
    int *flag;
    double qf, gqf;       // force charge and current weight
    double qx, gqx;       // second current over the same fields (second != 0)
    int first, sync, damp, accumulate, second;
};
struct LinkIO {
    const double *th;     // x_{n+1}
    double *thout;
    const double *kacc;
    const double *win;    // E
    double *wout, *sout;
    int *flag;
    int first, sync, damp;
};
int fabric_plan(int N, int nsm, ExtPlan *fabric, ExtPlan *second, ExtPlan *link);
cudaError_t fabric_step(const ExtPlan &plan, const FabConsts &c, const FabIO &io, cudaStream_t st);
cudaError_t link_step(const ExtPlan &plan, const FabConsts &c, const LinkIO &io, cudaStream_t st);

// Real mode with the optional terms: positions / momenta are 6 arrays (phi,
// theta); aux holds C and B (6 arrays) when the strain or hardening is on.
struct R6IO {
    const double *x;
    double *xout;
    const double *win;
    double *wout, *sout;
    double *aux;          // null: no strain or hardening term
    int *flag;
    int first, sync, damp;
};
int r6_plan(bool aux, int N, int nsm, ExtPlan *aux_plan, ExtPlan *step_plan);
cudaError_t r6_step(const ExtPlan &aux_plan, const ExtPlan &step_plan, const R6Consts &c, const R6IO &io,
                    cudaStream_t st);

// First diagnostics reduction of an FP64 state on the plane ring
// (diag_ring.cuh): 12 matter position arrays, the links and E (when the
// state carries them), the 12 matter momenta; one partial row per CTA.
struct DiagRingIO {
    const double *x[12];
    const double *th, *E;   // 3 arrays each, or null without links
    const double *mom;      // 12 arrays
};
int diag_ring_plan(bool gauged, bool links, int N, int nsm, ExtPlan *plan);
cudaError_t diag_ring_pass1(bool gauged, bool links, const ExtPlan &plan, const DiagConsts &c, const DiagRingIO &io,
                            double *part, cudaStream_t st);

}  // namespace scp
