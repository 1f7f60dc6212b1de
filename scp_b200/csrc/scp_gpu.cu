// scp_gpu.cu -- host side of the C ABI declared in include/scp_gpu.h.
//
// One handle = one simulation on one device with its own stream.  Device
// state (FP64 mode), each buffer NF = 12 (complex) or 15 (gauged) arrays of
// N^3 doubles, field-major, site index (i*N + j)*N + k:
//   X[0], X[1]  positions u v tu tv [th], double-buffered (stencil input and
//               output of the fused step)
//   W           half-step momenta w = v + hdt*a [and E + hdt*K], in place
//   S           synchronous momenta v [and E] of the last completed step
// After a scp_gpu_step call, X[cur^1] and S hold the state at the current
// time (what diagnostics and snapshots read) and X[cur], W the drifted
// positions and half-kicked momenta the next launch starts from.
//
// FP32-compensated mode keeps the same roles in FP32: positions as a
// pair X32[b] (fp32 hi) + LO[b] (bf16 lo of the 12 matter fields) + TLO[b]
// (fp32 lo of the 3 link angles), momenta W32, S32; the FP64 buffers
// only stage the initial state (and its Gauss projection) and are released.
#include "../../include/scp_gpu.h"
#include "common.cuh"
#include "diag.cuh"
#include "gauss.cuh"
#include "reduce.cuh"
#include "snapshot.cuh"
#include "spectral.cuh"
#include "launch.cuh"
#include "tma.cuh"
#include "ext_launch.cuh"
#include "ext_startup.cuh"

#include <cuda.h>   // driver API types only (entry points come through the runtime)
#include <nvtx3/nvToolsExt.h>   // header-only; ranges are free when no tool is attached
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <type_traits>
#include <mutex>

using namespace scp;

static thread_local char g_cuda_err[256] = "";

// NVTX range over one ABI call (init, step, diag, snapshot), so a timeline
// from a profiler shows the library's phases by name
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

#define CK(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            snprintf(g_cuda_err, sizeof g_cuda_err, "%s at %s:%d", cudaGetErrorString(e_), \
                     __FILE__, __LINE__);                                              \
            return e_ == cudaErrorMemoryAllocation ? SCP_ENOMEM : SCP_ECUDA;           \
        }                                                                              \
    } while (0)

namespace {

// FP32-compensated state from FP64 staging: hi = fp32(x), lo = bf16(x - hi),
// momenta fp32
__global__ void to_fp32c_kernel(const double *X, const double *S, int nf, long long n3, float *hi, uint16_t *lo,
                                float *tlo, float *S32) {
    const long long n = (long long)nf * n3;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double x = X[i];
        const float h = (float)x;
        const float l = (float)(x - (double)h);
        hi[i] = h;
        if (i < 12 * n3) lo[i] = f_to_bf16(l);
        else tlo[i - 12 * n3] = l;
        S32[i] = (float)S[i];
    }
}

// FP64 view of the FP32-compensated state for reductions and snapshots
struct View32C {
    const float *X;
    const uint16_t *LO;
    const float *TLO;
    const float *S;
    long long N3;
    __device__ __forceinline__ double q(int f, long long i) const {
        const float h = X[f * N3 + i];
        const float l = (f < 12) ? bf16_to_f(LO[f * N3 + i]) : TLO[(f - 12) * N3 + i];
        return (double)h + (double)l;
    }
    __device__ __forceinline__ double p(int f, long long i) const { return (double)S[f * N3 + i]; }
};

template <class View>
__global__ void extract_col_kernel(View V, int field, int mom, long long n, double *out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = mom ? V.p(field, i) : V.q(field, i);
}

}  // namespace

struct scp_gpu {
    scp_gpu_params p;
    StepConsts c;
    int N;
    long long N3;
    int gauged, nf, prec;
    int links;                   // th / E columns carried (complex_gauge; with g = 0 they stay constant)
    int real;                    // real 6-field mode: 12 host columns, imaginary sector held at zero
    // real 6-field mode with optional terms: ring kernels of real6.cuh; X[0..1],
    // W and S hold 6 arrays, raux the auxiliary C and B (strain, hardening)
    int rp = 0;
    double *raux = nullptr;
    R6Consts r6{};
    // gauged stepper with the Higgs condensate and/or the second gauge: one
    // fused ring kernel per step (higgs_u1.cuh); X[0..1], W and S hold nx arrays
    int gx = 0, g2 = 0, higgs = 0;
    HuConsts hc{};
    // three fabrics C, Q, L: one ring kernel per fabric and one for the links
    // per step (fabrics.cuh); X[0..1], W and S hold C (15), L (12), Q (12, free)
    int mfab = 0, fab_lock = 0;
    double qfab[3] = {0.0, 0.0, 0.0};
    FabConsts fc{};
    double *kacc = nullptr;      // accumulated currents (3 arrays)
    ExtPlan xplan{}, xplan2{}, lplan{};
    ExtPlan dplan{};             // first diagnostics reduction on the plane ring (FP64 states)
    int dplan_ok = 0;
    int nx = 0;                  // position arrays per buffer of the extension layouts
    int device;
    cudaStream_t stream = nullptr;
    // FP64 state
    double *slab = nullptr;
    double *X[2] = {nullptr, nullptr};
    double *W = nullptr, *S = nullptr;
    int cur = 0;
    // FP32-compensated state
    float *X32[2] = {nullptr, nullptr};
    uint16_t *LO[2] = {nullptr, nullptr};
    float *TLO[2] = {nullptr, nullptr};
    float *W32 = nullptr, *S32 = nullptr;
    void *slab32 = nullptr;
    // scratch
    double *part = nullptr, *fold = nullptr, *cg = nullptr, *point = nullptr;
    int *flag = nullptr;
    unsigned *count = nullptr;   // last-CTA counter of the fused CG launches
    double h_small[64];          // host landing area of the small device-to-host reads
    void *stage = nullptr;       // snapshot down-conversion staging (N3 doubles)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // asynchronous snapshots: device staging of every column, copies on their own stream
    cudaStream_t copy_stream = nullptr;
    void *snap_dev = nullptr;
    size_t snap_dev_bytes = 0;
    cudaEvent_t snap_ready = nullptr, snap_done = nullptr;
    int snap_pending = 0;
    // form of the FP64 fused step: 0 the cp.async ring, 1 TMA tile loads of
    // the positions (tensor maps of X[0], X[1]), 2 the cp.async ring with
    // TMA-staged momenta (tensor maps of W and S), 3 the gauged step with two
    // threads per site (step_duo.cuh)
    int tma = 0;
    // diagnostics summed by the synchronous FP64 step launch (classic form,
    // gauged or without links): per-CTA partials, the Gauss charge density,
    // and whether the partials describe the current state
    double *dpart = nullptr, *drho = nullptr;
    int dfuse = 0, dvalid = 0;
    TmaMaps tmaps[2];
    CUtensorMap mmaps[2];
    // launch geometry
    int shape;
    int pairs = 0;               // 1: two-site packed FP32C kernel
    int threads = 0;
    TileGrid tg;                 // item plan (the server's tables)
    int grid;
    TileGrid tg_run;             // plan of the single-grid launches (balanced when large enough)
    int grid_run = 0;
    int64_t steps = 0;
    double G_offset = 0.0;
    int cg_iters = 0;
    int64_t dev_bytes = 0;
};

static int validate(const scp_gpu_params *p) {
    if (!p) return SCP_EINVAL;
    if (p->N < 4 || p->N > 2048) return SCP_EINVAL;
    if (!(p->dx > 0) || !(p->dt > 0)) return SCP_EINVAL;
    if (p->complex_gauge && !(p->g_gauge >= 0)) return SCP_EINVAL;
    if (p->bc_type != 0 && p->bc_type != 2) return SCP_EUNSUPPORTED;
    if (p->precision_mode != SCP_PREC_FP64 && p->precision_mode != SCP_PREC_FP32C) return SCP_EINVAL;
    if (p->tile_variant < 0 || p->tile_variant >= kNumShapes) return SCP_EINVAL;
    if (p->real_fields != 0 && p->real_fields != 1) return SCP_EINVAL;
    if (p->real_fields && p->complex_gauge) return SCP_EUNSUPPORTED;   // links need the complex fields
    const bool optional = p->mode != 0 || p->alpha_cs != 0 || p->beta_h != 0 || p->kappa_h != 0;
    if (p->mode != 0 && p->mode != 1 && p->mode != 3) return SCP_EUNSUPPORTED;
    if (optional && !p->real_fields) return SCP_EINVAL;   // the reference allows them in the real mode only
    if (optional && p->precision_mode != SCP_PREC_FP64) return SCP_EUNSUPPORTED;
    // the reference ignores the gauged extensions without complex_gauge (scp_sim.c:229-238)
    if (p->complex_gauge && (p->higgs_v > 0 || p->g_gauge2 != 0)) {
        if (p->g_gauge == 0) return SCP_EUNSUPPORTED;   // the ungauged dispatch never evolves them
        if (p->precision_mode != SCP_PREC_FP64) return SCP_EUNSUPPORTED;
        if (!isfinite(p->g_gauge2) || !isfinite(p->higgs_v)) return SCP_EINVAL;
    }
    if (p->n_fabrics != 0 && p->n_fabrics != 1 && p->n_fabrics != 3) return SCP_EINVAL;
    if (p->n_fabrics == 3) {   // cfg_validate's rules (scp_config.h:518-534)
        if (!p->complex_gauge || p->real_fields) return SCP_EINVAL;
        if (p->higgs_v > 0 || p->g_gauge2 != 0) return SCP_EUNSUPPORTED;
        if (p->g_gauge == 0) return SCP_EUNSUPPORTED;   // the ungauged dispatch leaves Q and L unforced
        if (p->precision_mode != SCP_PREC_FP64) return SCP_EUNSUPPORTED;
    }
    return SCP_OK;
}

static void fill_consts(scp_gpu *h) {
    const scp_gpu_params &p = h->p;
    StepConsts &c = h->c;
    c.N = p.N;
    c.N3 = (long long)p.N * p.N * p.N;
    c.idx2 = 1.0 / (p.dx * p.dx);
    c.idx1 = 1.0 / (2.0 * p.dx);
    c.inva = 1.0 / p.dx;
    c.m2 = p.m2; c.mtheta2 = p.mtheta2; c.eta = p.eta; c.mu = p.mu; c.kappa = p.kappa;
    c.dt = p.dt;
    c.hdt = 0.5 * p.dt;
    const bool gauged = p.complex_gauge && p.g_gauge != 0.0;
    c.g = gauged ? p.g_gauge : 0.0;
    c.gad = -c.g * p.dx * p.dt;
    c.stp = gauged ? 1.0 / (p.g_gauge * p.dx * p.dx * p.dx) : 0.0;
    c.L = p.L; c.dx = p.dx;
    c.damp_width = p.damp_width;
    c.damp_rate = p.damp_rate;
    // next-plane momentum prefetch of the fused step (SCP_PREFETCH=0|1 in the
    // environment; off by default)
    const char *e = getenv("SCP_PREFETCH");
    c.prefetch = (e && e[0] == '1') ? 1 : 0;
    c.dV = p.dx * p.dx * p.dx;
    c.R2 = p.qdiag_radius * p.qdiag_radius;
    c.bpre = gauged ? 1.0 / (p.g_gauge * p.g_gauge * p.dx * p.dx * p.dx * p.dx) : 0.0;
}

static bool damping_on(const scp_gpu *h) {
    return h->p.bc_type == 0 && h->p.damp_width > 0 && h->p.damp_rate > 0;
}

// Choose the i-segment length that minimises (waves x planes per item),
// planes per item counting the two halo planes a segment re-reads.
static void plan_tiles(scp_gpu *h, int tx, int ty, int slots) {
    const int N = h->N;
    TileGrid tg;
    tg.ntx = (N + tx - 1) / tx;
    tg.nty = (N + ty - 1) / ty;
    const int ntiles = tg.ntx * tg.nty;

    double best = 1e300;
    int best_seg = N;
    const int cands[] = {4, 6, 8, 10, 12, 16, 20, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512, 1024, 2048};
    for (int s : cands) {
        if (s > N) break;
        const long long items = (long long)ntiles * ((N + s - 1) / s);
        const long long waves = (items + slots - 1) / slots;
        const double cost = (double)waves * (s + 2);
        if (cost < best - 1e-9 || (cost < best + 1e-9 && s > best_seg)) { best = cost; best_seg = s; }
    }
    {   // whole column as one segment
        const long long waves = (ntiles + slots - 1) / slots;
        const double cost = (double)waves * (N + 2);
        if (cost < best - 1e-9) { best = cost; best_seg = N; }
    }
    tg.seg = best_seg;
    tg.nseg = (N + best_seg - 1) / best_seg;
    tg.nitems = ntiles * tg.nseg;
    h->tg = tg;
    h->grid = tg.nitems < slots ? tg.nitems : slots;
    // All CTAs start their items on the same plane and walk i in step, so
    // neighbouring columns read each other's halo rows while they are in L2.
    // (Equal shares of all (column, plane) pairs, which leave no slot idle,
    // were measured slower: neighbours drift apart in i and the halo rows come
    // from DRAM again, 837 against 470 MB read per 128^3 step.)
    h->tg_run = tg;
    h->grid_run = h->grid;
}

template <class P>
static int occupancy_of(scp_gpu *h, int shape, int *occ) {
    size_t smem = 0;
    // raise the dynamic shared-memory cap of every variant of this shape
    for (int v = 0; v < 8; v++) {
        StepFnT<P> fn = step_fn<P>(shape, h->gauged, v & 1, (v >> 1) & 1, (v >> 2) & 1, &smem);
        CK(cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    StepFnT<P> fn = step_fn<P>(shape, h->gauged, false, false, false, &smem);
    const TileShape ts = kShapes[shape];
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, (const void *)fn, ts.tx * ts.ty, smem));
    return SCP_OK;
}

static int occupancy2_of(scp_gpu *h, int shape, int *occ) {
    size_t smem = 0;
    for (int v = 0; v < 8; v++) {
        StepFnT<F32C> fn = step2_fn(shape, h->gauged, v & 1, (v >> 1) & 1, (v >> 2) & 1, &smem);
        CK(cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    StepFnT<F32C> fn = step2_fn(shape, h->gauged, false, false, false, &smem);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, (const void *)fn, h->threads, smem));
    return SCP_OK;
}

// FP32C grids of even N run the two-site packed kernel; the default tile is
// 32 x 4 (one site per thread) and 32 x 8 (site pairs: 128 threads)
// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link libcuda)
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (EncodeTiledFn)f;
    }();
    return fn;
}

// The tensor maps of one FP64 position buffer (nf fields of N^3): a 4-D view
// (k, j, i, field) with boxes of TX x {TY+2, TY+1, 1} rows.  The buffer is the
// handle's own allocation on this device.
static bool encode_maps(const double *X, int N, int nf, int tx, int ty, TmaMaps *m) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t n = (cuuint64_t)N;
    const cuuint64_t dims[4] = {n, n, n, (cuuint64_t)nf};
    const cuuint64_t strides[3] = {n * 8, n * n * 8, n * n * n * 8};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUtensorMap *dst[3] = {&m->full, &m->part, &m->row};
    const cuuint32_t rows[3] = {(cuuint32_t)ty + 2, (cuuint32_t)ty + 1, 1};
    for (int q = 0; q < 3; q++) {
        const cuuint32_t box[4] = {(cuuint32_t)tx, rows[q], 1, 1};
        if (enc(dst[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)X, dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

// The tensor map of one FP64 momentum buffer: (k, j, i, field), box TX x TY.
static bool encode_mom_map(const double *W, int N, int nf, int tx, int ty, CUtensorMap *m) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t n = (cuuint64_t)N;
    const cuuint64_t dims[4] = {n, n, n, (cuuint64_t)nf};
    const cuuint64_t strides[3] = {n * 8, n * n * 8, n * n * n * 8};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const cuuint32_t box[4] = {(cuuint32_t)tx, (cuuint32_t)ty, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)W, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Staging of the FP64 step: the cp.async ring (0) by default.  The TMA forms
// apply to grids cut into full tiles, with a 16-byte row pitch and at least
// two tile rows along j, and are selected by SCP_STAGING in the environment:
// tma (1: TMA tile loads of the positions) or cpm (2: the cp.async position
// ring with TMA-staged momenta).  Both give the same bits as the default and
// ran slower on B200 (0.282 and 0.296 against 0.227 ms per 128^3 gauged
// step): the step is bound by shared-memory traffic and FP64 dependency
// chains, which the TMA forms do not shorten.
static int staging_mode(const scp_gpu *h, int shape) {
    if (h->prec != SCP_PREC_FP64 || (shape != 1 && shape != 2)) return 0;
    const char *e = getenv("SCP_STAGING");
    if (h->gauged && shape == 1 && e && strcmp(e, "duo") == 0) return 3;
    const TileShape ts = kShapes[shape];
    const int N = h->N;
    if (!(N % 2 == 0 && N % ts.tx == 0 && N % ts.ty == 0 && N >= 2 * ts.ty && N >= ts.tx)) return 0;
    if (e && strcmp(e, "tma") == 0) return 1;
    if (e && strcmp(e, "cpm") == 0) return 2;
    return 0;
}

// the two-threads-per-site kernels: shared-memory cap of every variant, and
// the CTAs of 2 x 32 x 4 threads one SM holds
static int setup_duo(scp_gpu *h, int *occ) {
    size_t smem = 0;
    for (int v = 0; v < 8; v++) {
        StepFnT<F64> fn = step_duo_fn(v & 1, (v >> 1) & 1, (v >> 2) & 1, &smem);
        CK(cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    StepFnT<F64> fn = step_duo_fn(false, false, false, &smem);
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, (const void *)fn, h->threads, smem));
    return SCP_OK;
}

static int setup_tma(scp_gpu *h, int *occ) {
    const TileShape ts = kShapes[h->shape];
    size_t smem = 0;
    const void *probe = nullptr;
    for (int v = 0; v < 8; v++) {
        const bool f = v & 1, sy = (v >> 1) & 1, d = (v >> 2) & 1;
        const void *fn = (h->tma == 1) ? (const void *)step_tma_fn(h->shape, h->gauged, f, sy, d, &smem)
                                       : (const void *)step_cpm_fn(h->shape, h->gauged, f, sy, d, &smem);
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (v == 0) probe = fn;
    }
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, probe, ts.tx * ts.ty, smem));
    if (h->tma == 1) {
        for (int b = 0; b < 2; b++)
            if (!encode_maps(h->X[b], h->N, h->nf, ts.tx, ts.ty, &h->tmaps[b])) return SCP_EUNSUPPORTED;
    } else {
        if (!encode_mom_map(h->W, h->N, h->nf, ts.tx, ts.ty, &h->mmaps[0]) ||
            !encode_mom_map(h->S, h->N, h->nf, ts.tx, ts.ty, &h->mmaps[1]))
            return SCP_EUNSUPPORTED;
    }
    return SCP_OK;
}

static int setup_launch(scp_gpu *h) {
    const bool pairs = h->prec == SCP_PREC_FP32C && h->N % 2 == 0;
    int shape = h->p.tile_variant;
    if (shape == 0) shape = pairs ? 2 : 1;
    h->shape = shape;
    h->pairs = pairs ? 1 : 0;
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    const TileShape ts = kShapes[shape];
    h->threads = ts.tx * ts.ty / (pairs ? 2 : 1);
    int occ = 0, rc;
    h->tma = staging_mode(h, shape);
    if (h->tma == 3) {
        h->threads = 2 * ts.tx * ts.ty;
        rc = setup_duo(h, &occ);
    } else if (h->tma) rc = setup_tma(h, &occ);
    else if (pairs) rc = occupancy2_of(h, shape, &occ);
    else if (h->prec == SCP_PREC_FP64) rc = occupancy_of<F64>(h, shape, &occ);
    else rc = occupancy_of<F32C>(h, shape, &occ);
    if (rc) return rc;
    if (occ < 1) return SCP_EUNSUPPORTED;
    plan_tiles(h, ts.tx, ts.ty, nsm * occ);
    return SCP_OK;
}

static int launch_step(scp_gpu *h, bool first, bool sync) {
    size_t smem = 0;
    const TileShape ts = kShapes[h->shape];
    if (h->prec == SCP_PREC_FP64) {
        StepIO<F64> io;
        io.xin = h->X[h->cur];
        io.xout = h->X[h->cur ^ 1];
        io.loin = nullptr;
        io.loout = nullptr;
        io.tloin = nullptr;
        io.tloout = nullptr;
        io.win = first ? h->S : h->W;
        io.wout = h->W;
        io.sout = h->S;
        io.flag = h->flag;
        const bool dg = sync && !first && h->dfuse;
        io.dpart = dg ? h->dpart : nullptr;
        io.drho = dg ? h->drho : nullptr;
        h->dvalid = dg ? 1 : 0;
        if (h->tma == 1) {
            TmaStepFn fn = step_tma_fn(h->shape, h->gauged, first, sync, damping_on(h), &smem);
            fn<<<h->grid_run, ts.tx * ts.ty, smem, h->stream>>>(io, h->c, h->tg_run, h->tmaps[h->cur]);
        } else if (h->tma == 2) {
            CpmStepFn fn = step_cpm_fn(h->shape, h->gauged, first, sync, damping_on(h), &smem);
            fn<<<h->grid_run, ts.tx * ts.ty, smem, h->stream>>>(io, h->c, h->tg_run, h->mmaps[first ? 1 : 0]);
        } else if (h->tma == 3) {
            StepFnT<F64> fn = step_duo_fn(first, sync, damping_on(h), &smem);
            fn<<<h->grid_run, h->threads, smem, h->stream>>>(io, h->c, h->tg_run);
        } else {
            StepFnT<F64> fn = step_fn<F64>(h->shape, h->gauged, first, sync, damping_on(h), &smem);
            fn<<<h->grid_run, ts.tx * ts.ty, smem, h->stream>>>(io, h->c, h->tg_run);
        }
    } else {
        StepIO<F32C> io;
        io.xin = h->X32[h->cur];
        io.xout = h->X32[h->cur ^ 1];
        io.loin = h->LO[h->cur];
        io.loout = h->LO[h->cur ^ 1];
        io.tloin = h->TLO[h->cur];
        io.tloout = h->TLO[h->cur ^ 1];
        io.win = first ? h->S32 : h->W32;
        io.wout = h->W32;
        io.sout = h->S32;
        io.flag = h->flag;
        h->dvalid = 0;
        if (h->pairs) {
            StepFnT<F32C> fn = step2_fn(h->shape, h->gauged, first, sync, damping_on(h), &smem);
            fn<<<h->grid_run, h->threads, smem, h->stream>>>(io, h->c, h->tg_run);
        } else {
            StepFnT<F32C> fn = step_fn<F32C>(h->shape, h->gauged, first, sync, damping_on(h), &smem);
            fn<<<h->grid_run, ts.tx * ts.ty, smem, h->stream>>>(io, h->c, h->tg_run);
        }
    }
    CK(cudaGetLastError());
    h->cur ^= 1;
    return SCP_OK;
}

// ---------------------------------------------------------------- Gauss law

static double fold_get(scp_gpu *h, int q) {   // after a synchronising copy
    return h->h_small[q];
}

static int fold_to_host(scp_gpu *h, int nq) {
    CK(cudaMemcpyAsync(h->h_small, h->fold, sizeof(double) * nq, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return SCP_OK;
}

static GaussArgs gauss_args(scp_gpu *h, const double *X, double *S) {
    GaussArgs a;
    a.X = X; a.S = S; a.N = h->N; a.N3 = h->N3; a.dx = h->p.dx; a.g = h->p.g_gauge;
    return a;
}

// net_charge_check + init_gauss_project on the state in (X, S)
constexpr int kCgItMax = 20000;   // init_gauss_project's iteration cap (scp_sim.c:2337)
constexpr int kCgBatch = 32;      // iterations enqueued between host checks

// Conjugate gradients on -lap(chi) = b - mean(b) (init_gauss_project's loop,
// scp_sim.c:2320-2372): b is in place and its block partial sums in h->part
// (nb blocks).  chi is left in x, less the xbar held in h->cg[CG_XBAR].
static int cg_solve(scp_gpu *h, int nb, double *b, double *x, double *r, double *p, double *Ap, int *iters) {
    const long long n3 = h->N3;
    const double n3d = (double)n3, idx2 = 1.0 / (h->p.dx * h->p.dx);
    fold_partials_kernel<1, 0><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
    cg_scalar_kernel<<<1, 1, 0, h->stream>>>(0, n3d, h->fold, h->cg);
    cg_start_kernel<<<nb, kRedThreads, 0, h->stream>>>(n3, b, r, p, x, h->cg, h->part);
    fold_partials_kernel<1, 1><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
    cg_scalar_kernel<<<1, 1, 0, h->stream>>>(1, n3d, h->fold, h->cg);
    CK(cudaGetLastError());
    if (spectral_supported(h->N)) {
        // start from the direct spectral solution of the same periodic 7-point
        // problem (spectral.cuh): r and p are its complex work arrays, then the
        // explicit residual of that chi restarts the iteration
        const int N = h->N, nc = spectral_ctas(N);
        const size_t sm = spectral_smem_bytes(N);
        CK(cudaFuncSetAttribute(is_pow2(N) ? (const void *)spectral_pass_kernel<true>
                                           : (const void *)spectral_pass_kernel<false>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        const double *in_re[5] = {b, r, r, r, r};
        const double *in_im[5] = {nullptr, p, p, p, p};
        double *out_re[5] = {r, r, r, r, x};
        double *out_im[5] = {p, p, p, p, nullptr};
        for (int pass = 0; pass < 5; pass++) {
            if (is_pow2(N))
                spectral_pass_kernel<true><<<nc, kFftThreads, sm, h->stream>>>(pass, N, idx2, in_re[pass],
                                                                               in_im[pass], out_re[pass],
                                                                               out_im[pass]);
            else
                spectral_pass_kernel<false><<<nc, kFftThreads, sm, h->stream>>>(pass, N, idx2, in_re[pass],
                                                                                in_im[pass], out_re[pass],
                                                                                out_im[pass]);
        }
        cg_warm_kernel<<<nb, kRedThreads, 0, h->stream>>>(N, n3, idx2, b, x, r, p, h->part);
        fold_partials_kernel<2, 1><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
        cg_scalar_kernel<<<1, 1, 0, h->stream>>>(2, n3d, h->fold, h->cg);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h->h_small, h->cg, sizeof(double) * CG_N, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (h->h_small[CG_DONE] != 0.0) {   // converged at the start: no iterations
            *iters = 0;
            return (h->h_small[CG_RMAX] > h->h_small[CG_TOL]) ? SCP_EGAUSS : SCP_OK;
        }
    }
    // the right-hand side is not needed any more: b is the second direction buffer
    double *dirs[2] = {p, b};
    // iterations in device-checked batches (see gauss.cuh); two launches each
    for (int batch = 0, it = 0;; batch++) {
        for (int k = 0; k < kCgBatch; k++, it++) {
            double *pold = dirs[it & 1], *pnew = dirs[(it + 1) & 1];
            cg_dirapply_kernel<<<nb, kRedThreads, 0, h->stream>>>(h->N, n3, idx2, r, pold, pnew, x, Ap, h->part,
                                                                  h->count, h->fold, h->cg);
            cg_update_kernel<<<nb, kRedThreads, 0, h->stream>>>(n3, x, r, pnew, Ap, h->part, h->count, h->fold,
                                                                h->cg, n3d, kCgItMax);
        }
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h->h_small, h->cg, sizeof(double) * CG_N, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (h->h_small[CG_DONE] != 0.0) break;
    }
    *iters = (int)h->h_small[CG_IT];
    return (h->h_small[CG_RMAX] > h->h_small[CG_TOL]) ? SCP_EGAUSS : SCP_OK;
}

static int gauss_startup(scp_gpu *h, const double *X, double *S) {
    const long long n3 = h->N3;
    const int nb = red_blocks(n3);
    GaussArgs a = gauss_args(h, X, S);
    const double dV = h->p.dx * h->p.dx * h->p.dx;
    int rc;
    if (h->p.bc_type == 2) {
        net_charge_kernel<<<nb, kRedThreads, 0, h->stream>>>(a, dV, h->part);
        fold_partials_kernel<2, 0><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
        CK(cudaGetLastError());
        if ((rc = fold_to_host(h, 2))) return rc;
        const double qn = fold_get(h, 0), qa = fold_get(h, 1);
        if (fabs(qn) > 1e-6 * fmax(qa, 1.0)) return SCP_ENETCHARGE;
    }
    if (!h->p.gauss_project) return SCP_OK;
    double *tmp = nullptr;
    CK(cudaMallocAsync(&tmp, sizeof(double) * 5 * n3, h->stream));
    double *b = tmp, *x = tmp + n3, *r = tmp + 2 * n3, *p = tmp + 3 * n3, *Ap = tmp + 4 * n3;
    gauss_rhs_kernel<<<nb, kRedThreads, 0, h->stream>>>(a, b, h->part);
    if ((rc = cg_solve(h, nb, b, x, r, p, Ap, &h->cg_iters))) {
        cudaFreeAsync(tmp, h->stream);
        return rc;
    }
    gauss_correct_kernel<<<nb, kRedThreads, 0, h->stream>>>(a, x, h->cg);
    gauss_sum_kernel<<<nb, kRedThreads, 0, h->stream>>>(a, h->part);
    fold_partials_kernel<1, 0><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
    CK(cudaGetLastError());
    CK(cudaFreeAsync(tmp, h->stream));
    if ((rc = fold_to_host(h, 1))) return rc;
    h->G_offset = fold_get(h, 0) / (double)n3;
    return SCP_OK;
}

// init_gauss2_project (scp_sim.c:2414-2458): the same solve for the second
// gauge's residual, correction into E2, no frozen offset
static int gauss2_startup(scp_gpu *h) {
    const long long n3 = h->N3;
    const int nb = red_blocks(n3);
    double *tmp = nullptr;
    CK(cudaMallocAsync(&tmp, sizeof(double) * 5 * n3, h->stream));
    double *b = tmp, *x = tmp + n3, *r = tmp + 2 * n3, *p = tmp + 3 * n3, *Ap = tmp + 4 * n3;
    double *E2 = h->S + (size_t)HiggsU1<false, true>::TH2 * n3;
    hu_gauss2_rhs_kernel<<<nb, kRedThreads, 0, h->stream>>>(h->X[0], h->S, E2, h->hc, b, h->part);
    int iters = 0, rc;
    if ((rc = cg_solve(h, nb, b, x, r, p, Ap, &iters))) {
        cudaFreeAsync(tmp, h->stream);
        return rc;
    }
    hu_gauss2_apply_kernel<<<nb, kRedThreads, 0, h->stream>>>(E2, x, h->cg, h->hc);
    CK(cudaGetLastError());
    CK(cudaFreeAsync(tmp, h->stream));
    return SCP_OK;
}

// ---------------------------------------------------------------- lifecycle

// Device memory comes from the device's default stream-ordered pool, kept
// instead of returned to the driver on synchronisation, so that handles made
// and freed at a high rate (the server) neither block nor re-map memory.
static std::once_flag g_pool_once[64];
static void keep_pool(int dev) {
    if (dev < 0 || dev >= 64) return;
    std::call_once(g_pool_once[dev], [dev] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    });
}

// Priority of the streams of handles created by this thread (0: default).  The
// server's loader threads raise it so that request start-up interleaves with
// the running chunks instead of queueing behind them.
static thread_local int t_stream_priority = 0;

static int alloc_common(scp_gpu *h) {
    keep_pool(h->device);
    CK(cudaStreamCreateWithPriority(&h->stream, cudaStreamNonBlocking, t_stream_priority));
    CK(cudaMallocAsync(&h->part, sizeof(double) * kRedMaxBlocks * 32, h->stream));
    CK(cudaMallocAsync(&h->fold, sizeof(double) * 64, h->stream));
    CK(cudaMallocAsync(&h->cg, sizeof(double) * 16, h->stream));
    CK(cudaMallocAsync(&h->point, sizeof(double) * 8, h->stream));
    CK(cudaMallocAsync(&h->flag, sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->flag, 0, sizeof(int), h->stream));
    CK(cudaMallocAsync(&h->count, sizeof(unsigned), h->stream));
    CK(cudaMemsetAsync(h->count, 0, sizeof(unsigned), h->stream));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    h->dev_bytes += sizeof(double) * (kRedMaxBlocks * 32 + 64 + 16 + 8);
    return SCP_OK;
}

static size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

static int init_body(scp_gpu *h, const double *const *cols, bool on_device) {
    int rc;
    if ((rc = alloc_common(h))) return rc;
    const long long n3 = h->N3;
    const int ncols = h->links ? 30 : 24;   // device columns (the real mode's imaginary ones are zero)
    const size_t nel = (size_t)h->nf * n3;
    const size_t blk = sizeof(double) * nel;
    // FP64 slab: X[0] = x_0 and S = v_0 stage the initial state in both modes;
    // FP64 mode also keeps X[1] and W in it
    const int nblk = (h->prec == SCP_PREC_FP64) ? 4 : 2;
    CK(cudaMallocAsync(&h->slab, nblk * blk, h->stream));
    h->dev_bytes += nblk * blk;
    h->X[0] = h->slab;
    h->S = h->slab + nel;
    if (h->prec == SCP_PREC_FP64) {
        h->X[1] = h->slab + 2 * nel;
        h->W = h->slab + 3 * nel;
    }
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int c = 0; c < ncols; c++) {
        int field, mom;
        sfa_col_source(c, &field, &mom);
        double *dst = (mom ? h->S : h->X[0]) + (size_t)field * n3;
        // real 6-field mode: the caller passes columns 0-11 only; v = tv = 0 exactly,
        // and the complex step keeps them zero (its real limit)
        cudaError_t e = (h->real && c >= 12) ? cudaMemsetAsync(dst, 0, sizeof(double) * n3, h->stream)
                                             : cudaMemcpyAsync(dst, cols[c], sizeof(double) * n3, kind, h->stream);
        if (e != cudaSuccess) {
            snprintf(g_cuda_err, sizeof g_cuda_err, "%s (column %d upload)", cudaGetErrorString(e), c);
            return SCP_ECUDA;
        }
    }
    if (h->gauged && (rc = gauss_startup(h, h->X[0], h->S))) return rc;
    // g = 0 with link columns: the ungauged step never writes th, so both
    // position buffers carry the same constant angles (E lives in S)
    if (h->links && !h->gauged && h->prec == SCP_PREC_FP64)
        CK(cudaMemcpyAsync(h->X[1] + (size_t)FTH * n3, h->X[0] + (size_t)FTH * n3, sizeof(double) * 3 * n3,
                           cudaMemcpyDeviceToDevice, h->stream));
    if ((rc = setup_launch(h))) return rc;
    CK(cudaMallocAsync(&h->stage, sizeof(double) * n3, h->stream));
    h->dev_bytes += sizeof(double) * n3;
    // the classic FP64 step sums the first diagnostics pass in its synchronous
    // launches (not with links at g = 0, whose step carries no th / E);
    // SCP_FUSED_DIAG=0 in the environment keeps the separate pass
    const char *fd = getenv("SCP_FUSED_DIAG");
    if (h->prec == SCP_PREC_FP64 && h->tma == 0 && (h->gauged || !h->links) && !(fd && fd[0] == '0')) {
        CK(cudaMallocAsync(&h->dpart, sizeof(double) * kDiag1Q * (size_t)h->grid_run, h->stream));
        h->dev_bytes += sizeof(double) * kDiag1Q * (size_t)h->grid_run;
        if (h->gauged) {
            CK(cudaMallocAsync(&h->drho, sizeof(double) * n3, h->stream));
            h->dev_bytes += sizeof(double) * n3;
        }
        h->dfuse = 1;
    }
    h->cur = 0;
    if (h->prec == SCP_PREC_FP64) return launch_step(h, true, false);
    // FP32-compensated buffers: X32[0..1], W32, S32 (fp32, NF arrays), LO[0..1]
    // (bf16, 12 arrays), TLO[0..1] (fp32, 3 arrays, gauged only)
    const size_t bf = round256(sizeof(float) * nel), bl = round256(sizeof(uint16_t) * 12 * (size_t)n3);
    const size_t bt = h->links ? round256(sizeof(float) * 3 * (size_t)n3) : 0;
    CK(cudaMallocAsync(&h->slab32, 4 * bf + 2 * bl + 2 * bt, h->stream));
    h->dev_bytes += 4 * bf + 2 * bl + 2 * bt;
    char *b = (char *)h->slab32;
    h->X32[0] = (float *)b; b += bf;
    h->X32[1] = (float *)b; b += bf;
    h->W32 = (float *)b; b += bf;
    h->S32 = (float *)b; b += bf;
    h->LO[0] = (uint16_t *)b; b += bl;
    h->LO[1] = (uint16_t *)b; b += bl;
    if (h->links) {
        h->TLO[0] = (float *)b; b += bt;
        h->TLO[1] = (float *)b;
    }
    to_fp32c_kernel<<<red_blocks((long long)nel), kRedThreads, 0, h->stream>>>(
        h->X[0], h->S, h->nf, n3, h->X32[0], h->LO[0], h->TLO[0], h->S32);
    CK(cudaGetLastError());
    if (h->links && !h->gauged) {   // constant angles in both position buffers (see above)
        CK(cudaMemcpyAsync(h->X32[1] + (size_t)FTH * n3, h->X32[0] + (size_t)FTH * n3, sizeof(float) * 3 * n3,
                           cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(h->TLO[1], h->TLO[0], sizeof(float) * 3 * n3, cudaMemcpyDeviceToDevice, h->stream));
    }
    if ((rc = launch_step(h, true, false))) return rc;
    // the FP64 staging is no longer needed: FP32C diagnostics read hi+lo directly
    CK(cudaFreeAsync(h->slab, h->stream));
    h->dev_bytes -= nblk * blk;
    h->slab = nullptr;
    h->X[0] = h->X[1] = h->W = h->S = nullptr;
    return SCP_OK;
}

// ---------------------------------------------------------------- real mode with optional terms

static bool real_optional(const scp_gpu_params *p) {
    return p->real_fields && (p->mode != 0 || p->alpha_cs != 0 || p->beta_h != 0 || p->kappa_h != 0);
}

static int ext_slab(scp_gpu *h, int nx);

// one step of the real mode: [auxiliary fields,] forces and fused leapfrog
static int r6_launch_step(scp_gpu *h, bool first, bool sync) {
    R6IO io;
    io.x = h->X[h->cur];
    io.xout = h->X[h->cur ^ 1];
    io.win = first ? h->S : h->W;
    io.wout = h->W;
    io.sout = h->S;
    io.aux = h->raux;
    io.flag = h->flag;
    io.first = first;
    io.sync = sync;
    io.damp = damping_on(h);
    CK(r6_step(h->xplan2, h->xplan, h->r6, io, h->stream));
    h->cur ^= 1;
    return SCP_OK;
}

static int init_real(scp_gpu *h, const double *const *cols, bool on_device) {
    int rc;
    if ((rc = alloc_common(h))) return rc;
    const long long n3 = h->N3;
    const scp_gpu_params &p = h->p;
    if ((rc = ext_slab(h, 6))) return rc;
    const bool aux = p.alpha_cs != 0 || p.beta_h != 0;
    if (aux) {
        CK(cudaMallocAsync(&h->raux, sizeof(double) * 6 * (size_t)n3, h->stream));
        CK(cudaMemsetAsync(h->raux, 0, sizeof(double) * 6 * (size_t)n3, h->stream));
        h->dev_bytes += sizeof(double) * 6 * n3;
    }
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int c = 0; c < 12; c++)   // phi, theta, then their velocities
        CK(cudaMemcpyAsync((c < 6 ? h->X[0] + c * n3 : h->S + (c - 6) * n3), cols[c], sizeof(double) * n3, kind,
                           h->stream));
    R6Consts &r = h->r6;
    r.N = p.N; r.N3 = n3; r.L = p.L; r.dx = p.dx; r.dV = p.dx * p.dx * p.dx;
    r.idx1 = 1.0 / (2.0 * p.dx); r.idx2 = 1.0 / (p.dx * p.dx); r.hdt = 0.5 * p.dt; r.dt = p.dt;
    r.mu = p.mu; r.kappa = p.kappa; r.m2 = p.m2; r.mtheta2 = p.mtheta2; r.eta = p.eta;
    r.kh = p.kappa_h; r.alpha = p.alpha_cs; r.beta = p.beta_h; r.kg = p.kappa_gamma;
    r.ia = p.inv_alpha; r.ib = p.inv_beta;
    r.mode = p.mode;
    r.damp_width = p.damp_width; r.damp_rate = p.damp_rate;
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    if (r6_plan(aux, h->N, nsm, &h->xplan2, &h->xplan)) return SCP_EUNSUPPORTED;
    return r6_launch_step(h, true, false);
}

static int real_diag(scp_gpu *h, scp_gpu_diag_out *out) {
    const int nb = red_blocks(h->N3);
    r6_energy_kernel<<<nb, kRedThreads, 0, h->stream>>>(h->X[h->cur ^ 1], h->S, h->r6, h->part);
    fold_partials_kernel<R6_NSUM, R6_NMAX><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_small, h->fold, sizeof(double) * (R6_NSUM + R6_NMAX), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const double *f = h->h_small;
    double *o = out->v;
    for (int q = 0; q < SCP_DIAG_NSLOTS; q++) o[q] = 0.0;
    const int slot[8] = {SCP_DIAG_E_PHI_KIN, SCP_DIAG_E_THETA_KIN, SCP_DIAG_E_GRAD, SCP_DIAG_E_MASS,
                         SCP_DIAG_E_POT, SCP_DIAG_E_TGRAD, SCP_DIAG_E_TMASS, SCP_DIAG_E_COUPLING};
    const int term[8] = {R6_EPK, R6_ETK, R6_EG, R6_EM, R6_EP, R6_ETG, R6_ETM, R6_EC};
    double total = 0.0;
    for (int q = 0; q < 8; q++) {
        o[slot[q]] = f[term[q]];
        total += f[term[q]];
    }
    o[SCP_DIAG_E_TOTAL] = total;
    o[SCP_DIAG_PHI_MAX] = f[R6_NSUM + R6_PHIMAX];
    o[SCP_DIAG_P_MAX] = f[R6_NSUM + R6_PMAX];
    o[SCP_DIAG_P_INT] = f[R6_PINT];
    o[SCP_DIAG_THETA_RMS] = sqrt(f[R6_TH2] / (3.0 * (double)h->N3));
    if (!isfinite(o[SCP_DIAG_E_TOTAL])) return SCP_ENONFINITE;
    return SCP_OK;
}

// ---------------------------------------------------------------- gauged extensions

static bool gext_on(const scp_gpu_params *p) {
    return p->complex_gauge && (p->higgs_v > 0 || p->g_gauge2 != 0);
}

// FP64 slab of the extension layouts: positions X[0], X[1], momenta W and
// the synchronous momenta S, nx arrays each
static int ext_slab(scp_gpu *h, int nx) {
    const size_t nel = (size_t)nx * h->N3;
    h->nx = nx;
    CK(cudaMallocAsync(&h->slab, sizeof(double) * 4 * nel, h->stream));
    CK(cudaMallocAsync(&h->stage, sizeof(double) * h->N3, h->stream));
    h->dev_bytes += sizeof(double) * (4 * nel + h->N3);
    CK(cudaMemsetAsync(h->slab, 0, sizeof(double) * 4 * nel, h->stream));
    h->X[0] = h->slab;
    h->X[1] = h->slab + nel;
    h->W = h->slab + 2 * nel;
    h->S = h->slab + 3 * nel;
    h->cur = 0;
    h->shape = 1;
    return SCP_OK;
}

// one step of the Higgs / second-gauge stepper: x_{n+1} in X[cur] -> X[cur^1]
static int hu_launch_step(scp_gpu *h, bool first, bool sync) {
    HuIO io;
    io.x = h->X[h->cur];
    io.xout = h->X[h->cur ^ 1];
    io.win = first ? h->S : h->W;
    io.wout = h->W;
    io.sout = h->S;
    io.flag = h->flag;
    io.first = first;
    io.sync = sync;
    io.damp = damping_on(h);
    CK(hu_step(h->higgs, h->g2, h->xplan, h->hc, io, h->stream));
    h->cur ^= 1;
    return SCP_OK;
}

static int init_gext(scp_gpu *h, const double *const *cols, bool on_device) {
    int rc;
    if ((rc = alloc_common(h))) return rc;
    const long long n3 = h->N3;
    const scp_gpu_params &p = h->p;
    h->g2 = p.g_gauge2 != 0 ? 1 : 0;
    h->higgs = p.higgs_v > 0 ? 1 : 0;
    if ((rc = ext_slab(h, 15 + 3 * h->g2 + h->higgs))) return rc;
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int c = 0; c < 30; c++) {   // th2, E2 start at zero
        int field, mom;
        sfa_col_source(c, &field, &mom);
        CK(cudaMemcpyAsync((mom ? h->S : h->X[0]) + (size_t)field * n3, cols[c], sizeof(double) * n3, kind,
                           h->stream));
    }
    HuConsts &k = h->hc;
    k.N = p.N; k.N3 = n3; k.L = p.L; k.dx = p.dx; k.dV = p.dx * p.dx * p.dx;
    k.idx1 = 1.0 / (2.0 * p.dx); k.idx2 = 1.0 / (p.dx * p.dx); k.inva = 1.0 / p.dx;
    k.hdt = 0.5 * p.dt; k.dt = p.dt;
    k.mu = p.mu; k.kappa = p.kappa; k.m2 = p.m2; k.mtheta2 = p.mtheta2; k.eta = p.eta;
    k.g = p.g_gauge;
    k.stp = 1.0 / (p.g_gauge * p.dx * p.dx * p.dx);
    k.gad = -p.g_gauge * p.dx * p.dt;
    k.g2 = p.g_gauge2;
    k.stp2 = h->g2 ? 1.0 / (p.g_gauge2 * p.dx * p.dx * p.dx) : 0.0;
    k.gad2 = -p.g_gauge2 * p.dx * p.dt;
    for (int a = 0; a < 3; a++) k.q[a] = p.gauge2_q[a];
    k.hv = p.higgs_v; k.hlam = p.higgs_lam; k.hkap = p.higgs_kap;
    k.damp_width = p.damp_width; k.damp_rate = p.damp_rate;
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    if (hu_plan(h->higgs, h->g2, h->N, nsm, &h->xplan)) return SCP_EUNSUPPORTED;
    // the reference's start-up order (scp_sim.c:2802-2836): Higgs start value,
    // net-charge check and Gauss projection, second Gauss projection, first force
    const int hf = 15 + 3 * h->g2;
    if (h->higgs)
        hu_higgs_start_kernel<<<red_blocks(n3), kRedThreads, 0, h->stream>>>(h->X[0] + (size_t)hf * n3,
                                                                              h->S + (size_t)hf * n3, k,
                                                                              p.higgs_rvoid);
    CK(cudaGetLastError());
    if ((rc = gauss_startup(h, h->X[0], h->S))) return rc;
    if (h->g2 && p.gauss_project && (rc = gauss2_startup(h))) return rc;
    return hu_launch_step(h, true, false);
}

// Higgs energy of the current state (the reference adds it to E_total, scp_sim.c:2034)
static int gext_higgs_energy(scp_gpu *h, double *e) {
    const int nb = red_blocks(h->N3);
    const size_t hf = (size_t)(15 + 3 * h->g2) * h->N3;
    const double *X = h->X[h->cur ^ 1];
    hu_higgs_energy_kernel<<<nb, kRedThreads, 0, h->stream>>>(X, X + hf, h->S + hf, h->hc, h->part);
    fold_partials_kernel<1, 0><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
    CK(cudaGetLastError());
    int rc;
    if ((rc = fold_to_host(h, 1))) return rc;
    *e = fold_get(h, 0);
    return SCP_OK;
}

// ---------------------------------------------------------------- three fabrics

static DiagConsts diag_consts(const scp_gpu *h);
template <class View>
static int diag_with(scp_gpu *h, const View &V, scp_gpu_diag_out *out);
static int diag_pass1_ring(scp_gpu *h, const DiagConsts &c, const double *Xm, const double *Pm, const double *th,
                           const double *E, int *rows);

// slots of the three-fabric layout
constexpr int kFabL = 15, kFabQ = 27;

// the fabrics at the time of buffers (X, P)
static FabView fab_view(const scp_gpu *h, const double *X, const double *P) {
    const size_t n3 = h->N3;
    FabView f;
    f.XC = X; f.PC = P;
    f.XL = X + kFabL * n3; f.PL = P + kFabL * n3;
    f.XQ = h->fab_lock ? X : X + kFabQ * n3;
    f.PQ = h->fab_lock ? P : P + kFabQ * n3;
    f.N3 = h->N3;
    for (int q = 0; q < 3; q++) f.q[q] = h->qfab[q];
    return f;
}

// one step of the three-fabric stepper: C (with the locked Q's force and
// currents), Q when free, L, then the links
static int fab_launch_step(scp_gpu *h, bool first, bool sync) {
    const size_t n3 = h->N3;
    const double *X = h->X[h->cur];
    double *Xo = h->X[h->cur ^ 1];
    const double *Win = first ? h->S : h->W;
    const double g = h->p.g_gauge;
    auto fabric = [&](size_t slot, double qf, bool second, double qx, bool acc) -> int {
        FabIO io;
        io.x = X + slot * n3;
        io.th = X + (size_t)FTH * n3;
        io.xout = Xo + slot * n3;
        io.win = Win + slot * n3;
        io.wout = h->W + slot * n3;
        io.sout = h->S + slot * n3;
        io.kacc = h->kacc;
        io.flag = h->flag;
        io.qf = qf;
        io.gqf = g * qf;
        io.qx = qx;
        io.gqx = g * qx;
        io.first = first;
        io.sync = sync;
        io.damp = damping_on(h);
        io.accumulate = acc;
        io.second = second;
        CK(fabric_step(second ? h->xplan2 : h->xplan, h->fc, io, h->stream));
        return SCP_OK;
    };
    int rc;
    const double qC = h->qfab[0], qQ = h->qfab[1], qL = h->qfab[2];
    if (h->fab_lock) {
        // C moves under the q_Q force; its q_C current precedes the q_Q one (none when q_C = 0)
        if ((rc = fabric(0, qQ, qC != 0.0, qC, false))) return rc;
    } else {
        if ((rc = fabric(0, qC, false, 0.0, false))) return rc;
        if ((rc = fabric(kFabQ, qQ, false, 0.0, true))) return rc;
    }
    if ((rc = fabric(kFabL, qL, false, 0.0, true))) return rc;
    LinkIO io;
    io.th = X + (size_t)FTH * n3;
    io.thout = Xo + (size_t)FTH * n3;
    io.kacc = h->kacc;
    io.win = Win + (size_t)FTH * n3;
    io.wout = h->W + (size_t)FTH * n3;
    io.sout = h->S + (size_t)FTH * n3;
    io.flag = h->flag;
    io.first = first;
    io.sync = sync;
    io.damp = damping_on(h);
    CK(link_step(h->lplan, h->fc, io, h->stream));
    h->cur ^= 1;
    return SCP_OK;
}

// the start-up of main with three fabrics (scp_sim.c:2818-2836): net-charge
// check and Gauss projection with rho_em, frozen offset
static int mf_gauss_startup(scp_gpu *h) {
    const long long n3 = h->N3;
    const int nb = red_blocks(n3);
    const FabView f = fab_view(h, h->X[0], h->S);
    const scp_gpu_params &p = h->p;
    int rc;
    if (p.bc_type == 2) {
        fabric_net_charge_kernel<<<nb, kRedThreads, 0, h->stream>>>(f, p.dx * p.dx * p.dx, h->part);
        fold_partials_kernel<2, 0><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
        CK(cudaGetLastError());
        if ((rc = fold_to_host(h, 2))) return rc;
        const double qn = fold_get(h, 0), qa = fold_get(h, 1);
        if (fabs(qn) > 1e-6 * fmax(qa, 1.0)) return SCP_ENETCHARGE;
    }
    if (!p.gauss_project) return SCP_OK;
    double *tmp = nullptr;
    CK(cudaMallocAsync(&tmp, sizeof(double) * 5 * n3, h->stream));
    double *b = tmp, *x = tmp + n3, *r = tmp + 2 * n3, *pp = tmp + 3 * n3, *Ap = tmp + 4 * n3;
    fabric_gauss_kernel<<<nb, kRedThreads, 0, h->stream>>>(f, h->N, p.dx, p.g_gauge, b, h->part);
    if ((rc = cg_solve(h, nb, b, x, r, pp, Ap, &h->cg_iters))) {
        cudaFreeAsync(tmp, h->stream);
        return rc;
    }
    gauss_correct_kernel<<<nb, kRedThreads, 0, h->stream>>>(gauss_args(h, h->X[0], h->S), x, h->cg);
    fabric_gauss_kernel<<<nb, kRedThreads, 0, h->stream>>>(f, h->N, p.dx, p.g_gauge, nullptr, h->part);
    fold_partials_kernel<1, 0><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
    CK(cudaGetLastError());
    CK(cudaFreeAsync(tmp, h->stream));
    if ((rc = fold_to_host(h, 1))) return rc;
    h->G_offset = fold_get(h, 0) / (double)n3;
    return SCP_OK;
}

static int init_mf(scp_gpu *h, const double *const *cols, bool on_device) {
    int rc;
    if ((rc = alloc_common(h))) return rc;
    const long long n3 = h->N3;
    const scp_gpu_params &p = h->p;
    h->fab_lock = p.mf_lock_CQ ? 1 : 0;
    for (int q = 0; q < 3; q++) h->qfab[q] = p.q_fab[q];
    if ((rc = ext_slab(h, h->fab_lock ? 27 : 39))) return rc;
    CK(cudaMallocAsync(&h->kacc, sizeof(double) * 3 * (size_t)n3, h->stream));
    h->dev_bytes += sizeof(double) * 3 * n3;
    // columns: C with the links (0-29), Q (30-53, skipped when locked), L (54-77)
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    for (int c = 0; c < 78; c++) {
        if (c >= 30 && c < 54 && h->fab_lock) continue;
        const int base = c < 30 ? 0 : (c < 54 ? 30 : 54);
        const size_t slot = base == 0 ? 0 : (base == 30 ? kFabQ : kFabL);
        int field, mom;
        sfa_col_source(c - base, &field, &mom);
        CK(cudaMemcpyAsync((mom ? h->S : h->X[0]) + (slot + field) * n3, cols[c], sizeof(double) * n3, kind,
                           h->stream));
    }
    FabConsts &k = h->fc;
    k.N = p.N; k.N3 = n3; k.L = p.L; k.dx = p.dx; k.dV = p.dx * p.dx * p.dx;
    k.idx1 = 1.0 / (2.0 * p.dx); k.idx2 = 1.0 / (p.dx * p.dx); k.inva = 1.0 / p.dx;
    k.hdt = 0.5 * p.dt; k.dt = p.dt;
    k.mu = p.mu; k.kappa = p.kappa; k.m2 = p.m2; k.mtheta2 = p.mtheta2; k.eta = p.eta;
    k.g = p.g_gauge;
    k.stp = 1.0 / (p.g_gauge * p.dx * p.dx * p.dx);
    k.gad = -p.g_gauge * p.dx * p.dt;
    k.damp_width = p.damp_width; k.damp_rate = p.damp_rate;
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    if (fabric_plan(h->N, nsm, &h->xplan, &h->xplan2, &h->lplan)) return SCP_EUNSUPPORTED;
    if ((rc = mf_gauss_startup(h))) return rc;
    return fab_launch_step(h, true, false);
}

// fabric C's diagnostics, plus fabric L's energies (compute_energy_complex_gauge,
// scp_sim.c:1977-2028), the Gauss norm with rho_em and the fabric charges
static int mf_diag(scp_gpu *h, scp_gpu_diag_out *out) {
    const double *X = h->X[h->cur ^ 1], *P = h->S;
    const size_t n3 = h->N3;
    ViewF64 V{X, P, h->N3};
    int rc = diag_with(h, V, out);
    if (rc && rc != SCP_ENONFINITE) return rc;
    const int nb = red_blocks(h->N3);
    const DiagConsts c = diag_consts(h);
    int nb1 = 0;
    if ((rc = diag_pass1_ring(h, c, X + kFabL * n3, P + kFabL * n3, X + FTH * n3, P + FTH * n3, &nb1))) return rc;
    fold_partials_kernel<DS_NSUM, DM_NMAX><<<1, 1024, 0, h->stream>>>(h->part, nb1, h->fold);
    CK(cudaGetLastError());
    if ((rc = fold_to_host(h, DS_EC + 1))) return rc;
    double *o = out->v;
    for (int q = 0; q <= DS_EC; q++) o[SCP_DIAG_E_PHI_KIN + q] += h->h_small[q];   // DS_EPK..DS_EC = slots 0..7
    o[SCP_DIAG_E_TOTAL] = o[SCP_DIAG_E_PHI_KIN] + o[SCP_DIAG_E_THETA_KIN] + o[SCP_DIAG_E_GRAD] + o[SCP_DIAG_E_MASS] +
                          o[SCP_DIAG_E_POT] + o[SCP_DIAG_E_TGRAD] + o[SCP_DIAG_E_TMASS] + o[SCP_DIAG_E_COUPLING] +
                          o[SCP_DIAG_E_EM];
    const scp_gpu_params &p = h->p;
    fabric_diag_kernel<<<nb, kRedThreads, 0, h->stream>>>(fab_view(h, X, P), h->N, p.L, p.dx, p.g_gauge, c.Rint2,
                                                          h->G_offset, h->part);
    fold_partials_kernel<FS_NSUM, 1><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold);
    CK(cudaGetLastError());
    if ((rc = fold_to_host(h, FS_NSUM + 1))) return rc;
    const double *f = h->h_small, dV = c.dV;
    o[SCP_DIAG_GAUSS_MAX] = f[FS_NSUM];
    o[SCP_DIAG_GAUSS_L2] = f[FS_NIN] > 0 ? sqrt(f[FS_GL2] / f[FS_NIN]) : 0.0;
    o[SCP_DIAG_Q_C] = f[FS_QC] * dV;
    o[SCP_DIAG_Q_Q] = f[FS_QQ] * dV;
    o[SCP_DIAG_Q_L] = f[FS_QL] * dV;
    o[SCP_DIAG_Q_EM] = f[FS_QEM] * dV;
    return isfinite(o[SCP_DIAG_E_TOTAL]) ? SCP_OK : SCP_ENONFINITE;
}

// columns of a snapshot: th2 and E2 follow the 30 gauged ones with the second
// gauge; fabric L's 24 with three fabrics
static int snap_ncols(const scp_gpu *h) {
    if (h->mfab) return 54;
    return h->links ? (h->g2 ? 36 : 30) : (h->real ? 12 : 24);
}

// source of host column c: the packed arrays it lives in (positions, momenta)
// and its slot there
static void col_source(const scp_gpu *h, int c, const double **X, const double **S, int *field, int *mom) {
    *X = h->X[h->cur ^ 1];
    *S = h->S;
    if (h->rp) { *field = c % 6; *mom = c >= 6; return; }   // the 6-field layout
    if (c >= 30 && h->g2) {                                 // th2 / E2 after the 15-field block
        *field = 15 + (c - 30) % 3; *mom = c >= 33;
        return;
    }
    if (c >= 30 && h->mfab) {                               // fabric L after C
        sfa_col_source(c - 30, field, mom);
        *field += kFabL;
        return;
    }
    sfa_col_source(c, field, mom);
}

static int init_common(const scp_gpu_params *p, const double *const *cols, bool on_device, scp_gpu **out) {
    if (!out) return SCP_EINVAL;
    *out = nullptr;
    int rc = validate(p);
    if (rc) return rc;
    if (!cols) return SCP_EINVAL;
    const int ncols = p->n_fabrics == 3 ? 78 : (p->complex_gauge ? 30 : (p->real_fields ? 12 : 24));
    for (int c = 0; c < ncols; c++)
        if (!cols[c] && !(c >= 30 && c < 54 && p->n_fabrics == 3 && p->mf_lock_CQ)) return SCP_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= p->device || p->device < 0) return SCP_ENODEV;
    CK(cudaSetDevice(p->device));
    scp_gpu *h = new scp_gpu();
    h->p = *p;
    h->device = p->device;
    h->N = p->N;
    h->N3 = (long long)p->N * p->N * p->N;
    // the reference dispatches on complex_gauge && g != 0 (scp_sim.c:1586, :2820):
    // with g = 0 it runs the ungauged dynamics and carries th / E unchanged
    h->links = p->complex_gauge ? 1 : 0;
    h->real = p->real_fields ? 1 : 0;
    h->gauged = (p->complex_gauge && p->g_gauge != 0.0) ? 1 : 0;
    h->nf = h->links ? 15 : 12;
    h->prec = p->precision_mode;
    fill_consts(h);
    h->rp = real_optional(p) ? 1 : 0;
    h->gx = gext_on(p) ? 1 : 0;
    h->mfab = p->n_fabrics == 3 ? 1 : 0;
    if (h->rp) rc = init_real(h, cols, on_device);
    else if (h->gx) rc = init_gext(h, cols, on_device);
    else if (h->mfab) rc = init_mf(h, cols, on_device);
    else rc = init_body(h, cols, on_device);
    if (rc == SCP_OK) {
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) {
            snprintf(g_cuda_err, sizeof g_cuda_err, "%s (init)", cudaGetErrorString(e));
            rc = SCP_ECUDA;
        }
    }
    if (rc) {
        scp_gpu_free(h);
        return rc;
    }
    *out = h;
    return SCP_OK;
}

extern "C" {

int scp_gpu_init(const scp_gpu_params *p, const double *const *host_cols, scp_gpu **out) {
    NvtxRange range_("scp_gpu_init");
    return init_common(p, host_cols, false, out);
}

int scp_gpu_init_device(const scp_gpu_params *p, const double *const *dev_cols, scp_gpu **out) {
    NvtxRange range_("scp_gpu_init_device");
    return init_common(p, dev_cols, true, out);
}

int scp_gpu_step(scp_gpu *h, int nsteps) {
    NvtxRange range_("scp_gpu_step");
    if (!h || nsteps < 0) return SCP_EINVAL;
    if (nsteps == 0) return SCP_OK;
    CK(cudaSetDevice(h->device));
    int rc;
    if (h->gx || h->mfab) {
        for (int n = 0; n < nsteps; n++) {
            const bool last = (n == nsteps - 1);
            if ((rc = h->gx ? hu_launch_step(h, false, last) : fab_launch_step(h, false, last))) return rc;
        }
        h->steps += nsteps;
        return SCP_OK;
    }
    if (h->rp) {
        for (int n = 0; n < nsteps; n++)
            if ((rc = r6_launch_step(h, false, n == nsteps - 1))) return rc;
        h->steps += nsteps;
        return SCP_OK;
    }
    for (int n = 0; n < nsteps; n++) {
        const bool last = (n == nsteps - 1);
        if ((rc = launch_step(h, false, last))) return rc;
    }
    h->steps += nsteps;
    return SCP_OK;
}

int scp_gpu_sync(scp_gpu *h) {
    if (!h) return SCP_EINVAL;
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->h_small, h->flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    int f = 0;
    memcpy(&f, h->h_small, sizeof(int));
    if (f & kFlagTimeout) return SCP_ETIMEOUT;
    return f ? SCP_ENONFINITE : SCP_OK;
}

}  // extern "C"

// Diagnostic slots from the folded reductions: f1 = pass-1 sums then maxima,
// f2 = pass-2 sums, pt = point values (omega_core, theta probes).
static void diag_assemble(const double *f1, const double *f2, const double *pt, const DiagConsts &c,
                          long long n3, double g_gauge, scp_gpu_diag_out *out) {
    const double dV = c.dV;
    double *o = out->v;
    for (int q = 0; q < SCP_DIAG_NSLOTS; q++) o[q] = 0.0;
    o[SCP_DIAG_E_PHI_KIN] = f1[DS_EPK];
    o[SCP_DIAG_E_THETA_KIN] = f1[DS_ETK];
    o[SCP_DIAG_E_GRAD] = f1[DS_EG];
    o[SCP_DIAG_E_MASS] = f1[DS_EM];
    o[SCP_DIAG_E_POT] = f1[DS_EP];
    o[SCP_DIAG_E_TGRAD] = f1[DS_ETG];
    o[SCP_DIAG_E_TMASS] = f1[DS_ETM];
    o[SCP_DIAG_E_COUPLING] = f1[DS_EC];
    // the gauged energy counts E_em (compute_energy_complex_gauge); with g = 0 the
    // reference evaluates the ungauged energy and reports E_em separately
    o[SCP_DIAG_E_TOTAL] = f1[DS_EPK] + f1[DS_ETK] + f1[DS_EG] + f1[DS_EM] + f1[DS_EP] + f1[DS_ETG] +
                          f1[DS_ETM] + f1[DS_EC] + (c.gauged ? f1[DS_EEM] : 0.0);
    o[SCP_DIAG_PHI_MAX] = f1[DS_NSUM + DM_PM];
    o[SCP_DIAG_P_MAX] = f1[DS_NSUM + DM_PMAX];
    o[SCP_DIAG_P_INT] = f1[DS_PINT];
    // complex: over 6 real components per site (theta_rms_complex); real mode: over
    // the 3 real angles (theta_rms, scp_sim.c:1803-1809), the imaginary parts being zero
    o[SCP_DIAG_THETA_RMS] = sqrt(f1[DS_TRS] / ((c.real ? 3.0 : 6.0) * (double)n3));
    o[SCP_DIAG_Q_PHI] = f1[DS_QP] * dV;
    o[SCP_DIAG_Q_THETA] = f1[DS_QT] * dV;
    o[SCP_DIAG_Q_TOTAL] = f1[DS_QP] * dV + f1[DS_QT] * dV;
    o[SCP_DIAG_S_MAX] = f1[DS_NSUM + DM_SMAX];
    const double M0 = f1[DS_M0] * dV;
    o[SCP_DIAG_R_CORE] = (M0 < 1e-30) ? 0.0 : sqrt(f2[0] * dV / M0);
    o[SCP_DIAG_OMEGA_CORE] = pt[0];
    o[SCP_DIAG_Q_CORE] = f1[DS_QC] * dV;
    o[SCP_DIAG_THP1U] = pt[1]; o[SCP_DIAG_THP1V] = pt[2];
    o[SCP_DIAG_THP2U] = pt[3]; o[SCP_DIAG_THP2V] = pt[4];
    if (c.links) {   // compute_gauss (scp_sim.c:2186-2243)
        o[SCP_DIAG_GAUSS_MAX] = f1[DS_NSUM + DM_GMAX];
        o[SCP_DIAG_GAUSS_L2] = f1[DS_NOM] > 0 ? sqrt(f1[DS_GL2] / f1[DS_NOM]) : 0.0;
        o[SCP_DIAG_E_EM] = f1[DS_EEM];
        o[SCP_DIAG_Q_FLUX] = (g_gauge != 0.0) ? (f1[DS_FSUM] - c.G_offset * f1[DS_NC] * dV) / g_gauge : 0.0;
    }
    o[SCP_DIAG_Q_P0] = f1[DS_QP0] * dV;
    o[SCP_DIAG_Q_P1] = f1[DS_QP1] * dV;
    o[SCP_DIAG_Q_P2] = f1[DS_QP2] * dV;
    if (!(M0 < 1e-30)) {
        o[SCP_DIAG_CENTROID_X] = f1[DS_CX] * dV / M0;
        o[SCP_DIAG_CENTROID_Y] = f1[DS_CY] * dV / M0;
        o[SCP_DIAG_CENTROID_Z] = f1[DS_CZ] * dV / M0;
    }
}

// Reduction constants of a state on grid p: the one place DiagConsts is
// filled, for the handle diagnostics and for scp_gpu_diag_noalloc alike.
static DiagConsts diag_consts_for(const scp_gpu_params &p, int gauged, int links, int real, double G_offset) {
    DiagConsts c;
    c.N = p.N; c.N3 = (long long)p.N * p.N * p.N; c.L = p.L; c.dx = p.dx; c.dV = p.dx * p.dx * p.dx;
    c.idx1 = 1.0 / (2.0 * p.dx);
    c.m2 = p.m2; c.mtheta2 = p.mtheta2; c.eta = p.eta; c.mu = p.mu; c.kappa = p.kappa;
    c.gauged = gauged;
    c.links = links;
    c.real = real;
    c.g = gauged ? p.g_gauge : 0.0;
    c.bpre = gauged ? 1.0 / (p.g_gauge * p.g_gauge * p.dx * p.dx * p.dx * p.dx) : 0.0;
    c.R2 = p.qdiag_radius * p.qdiag_radius;
    c.Rcube = p.qdiag_radius;
    const double Rint = (p.bc_type == 0) ? (p.L - p.damp_width - p.dx) : 1e300;
    c.Rint2 = Rint * Rint;
    c.G_offset = G_offset;
    return c;
}

static DiagConsts diag_consts(const scp_gpu *h) {
    return diag_consts_for(h->p, h->gauged, h->links, h->real, h->G_offset);
}

// First diagnostics reduction of an FP64 state on the plane ring: matter
// positions Xm and momenta Pm (12 arrays each), links and E (3 each, or null);
// the partial rows land in h->part, their count in *rows.
static int diag_pass1_ring(scp_gpu *h, const DiagConsts &c, const double *Xm, const double *Pm, const double *th,
                           const double *E, int *rows) {
    if (!h->dplan_ok) {
        int nsm = 0;
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
        if (diag_ring_plan(c.gauged, c.links, h->N, nsm, &h->dplan)) return SCP_EUNSUPPORTED;
        h->dplan_ok = 1;
    }
    DiagRingIO io;
    for (int f = 0; f < 12; f++) io.x[f] = Xm + (size_t)f * h->N3;
    io.th = th;
    io.E = E;
    io.mom = Pm;
    CK(diag_ring_pass1(c.gauged, c.links, h->dplan, c, io, h->part, h->stream));
    *rows = h->dplan.grid;
    return SCP_OK;
}

template <class View>
static int diag_with(scp_gpu *h, const View &V, scp_gpu_diag_out *out) {
    const scp_gpu_params &p = h->p;
    const DiagConsts c = diag_consts(h);
    const int nb = red_blocks(h->N3);
    int nb1 = nb;
    const double *part1 = h->part;
    // pass 1 already summed by the synchronous step launch that produced this state
    const bool fused = std::is_same<View, ViewF64>::value && h->dvalid;
    if constexpr (std::is_same<View, ViewF64>::value) {
        if (fused) {
            nb1 = h->grid_run;
            part1 = h->dpart;
        } else {
            const size_t th = (size_t)FTH * h->N3;
            int rc = diag_pass1_ring(h, c, V.X, V.S, c.links ? V.X + th : nullptr, c.links ? V.S + th : nullptr,
                                     &nb1);
            if (rc) return rc;
        }
    } else {
        diag_pass1_kernel<View><<<nb, kRedThreads, 0, h->stream>>>(V, c, h->part);
    }
    fold_partials_kernel<DS_NSUM, DM_NMAX><<<1, 1024, 0, h->stream>>>(part1, nb1, h->fold);
    // pass 2 (r_core, argmax site), with the Gauss-law slots when pass 1 was fused
    const bool gauss2 = fused && c.links;
    const double *negidx;
    if (gauss2) {
        diag_pass2g_kernel<View><<<nb, kRedThreads, 0, h->stream>>>(V, c, h->fold, h->drho, h->part);
        fold_partials_kernel<5, 2><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold + 44);
        negidx = h->fold + 49;
    } else {
        diag_pass2_kernel<View><<<nb, kRedThreads, 0, h->stream>>>(V, c, h->fold, h->part);
        fold_partials_kernel<1, 1><<<1, 1024, 0, h->stream>>>(h->part, nb, h->fold + 40);
        negidx = h->fold + 41;
    }
    diag_point_kernel<View><<<1, 32, 0, h->stream>>>(V, c, negidx, p.qdiag_probe1, p.qdiag_probe2, h->point);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h->h_small, h->fold, sizeof(double) * 51, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->h_small + 56, h->point, sizeof(double) * 5, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double f1[kDiag1Q], f2[2] = {h->h_small[40], h->h_small[41]};
    memcpy(f1, h->h_small, sizeof f1);
    if (gauss2) {   // [rsum, GL2, NOM, FSUM, NC | -min_idx, GMAX]
        const double *g = h->h_small + 44;
        f2[0] = g[0];
        f2[1] = g[5];
        f1[DS_GL2] = g[1];
        f1[DS_NOM] = g[2];
        f1[DS_FSUM] = g[3];
        f1[DS_NC] = g[4];
        f1[DS_NSUM + DM_GMAX] = g[6];
    }
    diag_assemble(f1, f2, h->h_small + 56, c, h->N3, p.g_gauge, out);
    if (!isfinite(out->v[SCP_DIAG_E_TOTAL])) return SCP_ENONFINITE;
    return SCP_OK;
}

extern "C" {

int scp_gpu_diag(scp_gpu *h, scp_gpu_diag_out *out) {
    NvtxRange range_("scp_gpu_diag");
    if (!h || !out) return SCP_EINVAL;
    CK(cudaSetDevice(h->device));
    if (h->rp) return real_diag(h, out);
    if (h->mfab) return mf_diag(h, out);
    if (h->gx) {
        ViewF64 V{h->X[h->cur ^ 1], h->S, h->N3};
        int rc = diag_with(h, V, out);
        if (rc || !h->higgs) return rc;
        double eh = 0.0;
        if ((rc = gext_higgs_energy(h, &eh))) return rc;
        out->v[SCP_DIAG_E_TOTAL] += eh;
        return isfinite(out->v[SCP_DIAG_E_TOTAL]) ? SCP_OK : SCP_ENONFINITE;
    }
    if (h->prec == SCP_PREC_FP64) {
        ViewF64 V{h->X[h->cur ^ 1], h->S, h->N3};
        return diag_with(h, V, out);
    }
    View32C V{h->X32[h->cur ^ 1], h->LO[h->cur ^ 1], h->TLO[h->cur ^ 1], h->S32, h->N3};
    return diag_with(h, V, out);
}

}  // extern "C"

// one SFA column of the current state, converted to the snapshot dtype, into
// the staging buffer (the f16 rule is the reference's, snapshot.cuh)
template <class View>
__global__ void snap_col_kernel(View V, int field, int mom, long long n, int dtype, void *out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = mom ? V.p(field, i) : V.q(field, i);
        if (dtype == SCP_DTYPE_F64) ((double *)out)[i] = v;
        else if (dtype == SCP_DTYPE_F32) ((float *)out)[i] = (float)v;
        else ((uint16_t *)out)[i] = f64_to_f16_trunc(v);
    }
}

template <class View>
static int snapshot_with(scp_gpu *h, const View &V, int dtype, void *const *host_cols) {
    const int ncols = snap_ncols(h);
    const long long n3 = h->N3;
    const int nb = red_blocks(n3);
    const size_t es = dtype == SCP_DTYPE_F64 ? 8 : (dtype == SCP_DTYPE_F32 ? 4 : 2);
    for (int c = 0; c < ncols; c++) {
        if (!host_cols[c]) return SCP_EINVAL;
        const double *Xs, *Ss;
        int field, mom;
        col_source(h, c, &Xs, &Ss, &field, &mom);
        if (h->prec == SCP_PREC_FP64 && dtype == SCP_DTYPE_F64) {   // straight copy of the FP64 column
            const double *src = (mom ? Ss : Xs) + (size_t)field * n3;
            CK(cudaMemcpyAsync(host_cols[c], src, sizeof(double) * n3, cudaMemcpyDeviceToHost, h->stream));
        } else {
            if (h->prec == SCP_PREC_FP64) {
                ViewF64 V2{Xs, Ss, n3};
                snap_col_kernel<ViewF64><<<nb, kRedThreads, 0, h->stream>>>(V2, field, mom, n3, dtype, h->stage);
            } else {
                snap_col_kernel<View><<<nb, kRedThreads, 0, h->stream>>>(V, field, mom, n3, dtype, h->stage);
            }
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(host_cols[c], h->stage, es * n3, cudaMemcpyDeviceToHost, h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));   // staging buffer reused per column
    }
    return SCP_OK;
}

extern "C" {

int scp_gpu_snapshot(scp_gpu *h, int dtype, void *const *host_cols) {
    NvtxRange range_("scp_gpu_snapshot");
    if (!h || !host_cols) return SCP_EINVAL;
    if (dtype != SCP_DTYPE_F16 && dtype != SCP_DTYPE_F32 && dtype != SCP_DTYPE_F64) return SCP_EINVAL;
    CK(cudaSetDevice(h->device));
    if (h->prec == SCP_PREC_FP64) {
        ViewF64 V{h->X[h->cur ^ 1], h->S, h->N3};
        return snapshot_with(h, V, dtype, host_cols);
    }
    View32C V{h->X32[h->cur ^ 1], h->LO[h->cur ^ 1], h->TLO[h->cur ^ 1], h->S32, h->N3};
    return snapshot_with(h, V, dtype, host_cols);
}

}  // extern "C"

// Down-convert every column of the current state into device staging on the
// handle's stream (later steps overwrite the state, so this part is ordered
// with them), then copy the staging to the host on the copy stream.
template <class View>
static int snapshot_async_with(scp_gpu *h, const View &V, int dtype, void *const *host_cols) {
    const int ncols = snap_ncols(h);
    const long long n3 = h->N3;
    const size_t es = dtype == SCP_DTYPE_F64 ? 8 : (dtype == SCP_DTYPE_F32 ? 4 : 2);
    const size_t col = es * (size_t)n3, need = col * ncols;
    for (int c = 0; c < ncols; c++)
        if (!host_cols[c]) return SCP_EINVAL;
    if (!h->copy_stream) {
        CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&h->snap_ready, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->snap_done, cudaEventDisableTiming));
    }
    if (h->snap_dev_bytes < need) {
        if (h->snap_dev) {
            CK(cudaFreeAsync(h->snap_dev, h->stream));
            h->dev_bytes -= h->snap_dev_bytes;
            h->snap_dev = nullptr;
            h->snap_dev_bytes = 0;
        }
        CK(cudaMallocAsync(&h->snap_dev, need, h->stream));
        h->snap_dev_bytes = need;
        h->dev_bytes += need;
    }
    char *stage = (char *)h->snap_dev;
    const int nb = red_blocks(n3);
    for (int c = 0; c < ncols; c++) {
        const double *Xs, *Ss;
        int field, mom;
        col_source(h, c, &Xs, &Ss, &field, &mom);
        if (h->prec == SCP_PREC_FP64 && dtype == SCP_DTYPE_F64) {
            const double *src = (mom ? Ss : Xs) + (size_t)field * n3;
            CK(cudaMemcpyAsync(stage + c * col, src, col, cudaMemcpyDeviceToDevice, h->stream));
        } else if (h->prec == SCP_PREC_FP64) {
            ViewF64 V2{Xs, Ss, n3};
            snap_col_kernel<ViewF64><<<nb, kRedThreads, 0, h->stream>>>(V2, field, mom, n3, dtype, stage + c * col);
        } else {
            snap_col_kernel<View><<<nb, kRedThreads, 0, h->stream>>>(V, field, mom, n3, dtype, stage + c * col);
        }
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(h->snap_ready, h->stream));
    CK(cudaStreamWaitEvent(h->copy_stream, h->snap_ready, 0));
    for (int c = 0; c < ncols; c++)
        CK(cudaMemcpyAsync(host_cols[c], stage + c * col, col, cudaMemcpyDeviceToHost, h->copy_stream));
    CK(cudaEventRecord(h->snap_done, h->copy_stream));
    h->snap_pending = 1;
    return SCP_OK;
}

extern "C" {

int scp_gpu_snapshot_wait(scp_gpu *h) {
    if (!h) return SCP_EINVAL;
    if (!h->snap_pending) return SCP_OK;
    CK(cudaSetDevice(h->device));
    h->snap_pending = 0;
    CK(cudaEventSynchronize(h->snap_done));
    return SCP_OK;
}

int scp_gpu_snapshot_async(scp_gpu *h, int dtype, void *const *host_cols) {
    NvtxRange range_("scp_gpu_snapshot_async");
    if (!h || !host_cols) return SCP_EINVAL;
    if (dtype != SCP_DTYPE_F16 && dtype != SCP_DTYPE_F32 && dtype != SCP_DTYPE_F64) return SCP_EINVAL;
    int rc;
    if ((rc = scp_gpu_snapshot_wait(h))) return rc;   // one snapshot in flight per handle
    CK(cudaSetDevice(h->device));
    if (h->prec == SCP_PREC_FP64) {
        ViewF64 V{h->X[h->cur ^ 1], h->S, h->N3};
        return snapshot_async_with(h, V, dtype, host_cols);
    }
    View32C V{h->X32[h->cur ^ 1], h->LO[h->cur ^ 1], h->TLO[h->cur ^ 1], h->S32, h->N3};
    return snapshot_async_with(h, V, dtype, host_cols);
}

void *scp_gpu_host_alloc(size_t bytes) {
    void *p = nullptr;
    if (cudaMallocHost(&p, bytes) != cudaSuccess) return nullptr;
    return p;
}

void scp_gpu_host_free(void *p) {
    if (p) cudaFreeHost(p);
}

int scp_gpu_get_info(const scp_gpu *h, scp_gpu_info *info) {
    if (!h || !info) return SCP_EINVAL;
    memset(info, 0, sizeof *info);
    info->steps_done = h->steps;
    info->time = (double)h->steps * h->p.dt;
    info->G_offset = h->G_offset;
    info->cg_iterations = h->cg_iters;
    info->precision_mode = h->prec;
    info->device_bytes = h->dev_bytes;
    // persistent bytes per site the step reads and writes: x and w (FP64);
    // hi (fp32) + lo (bf16 matter, fp32 links) + w (fp32) in FP32C
    // (the fields the step touches: 15 gauged, 12 otherwise, links carried
    // unchanged with g = 0 included in neither)
    const double nfs = h->gauged ? 15.0 : 12.0;
    info->state_bytes_per_site = (h->prec == SCP_PREC_FP64)
                                     ? 2.0 * 8.0 * nfs
                                     : 4.0 * nfs + 12.0 * 2.0 + (h->gauged ? 3.0 * 4.0 : 0.0) + 4.0 * nfs;
    // extensions: positions and momenta (30), th2 / E2 (6), H / Hdot (2), FP64
    if (h->gx) info->state_bytes_per_site = 8.0 * (30.0 + 6.0 * h->g2 + 2.0 * h->higgs);
    // three fabrics: C with the links (30), L (24), Q (24) unless it is C
    if (h->mfab) info->state_bytes_per_site = 8.0 * (30.0 + 24.0 + (h->fab_lock ? 0.0 : 24.0));
    info->step_bytes_per_site = 2.0 * info->state_bytes_per_site;
    info->tile_x = kShapes[h->shape].tx;
    info->tile_y = kShapes[h->shape].ty;
    info->seg_len = h->tg_run.seg;
    info->sites_per_thread = h->pairs ? 2 : 1;
    info->tma_staging = h->tma;
    return SCP_OK;
}

int scp_gpu_time_steps(scp_gpu *h, int nsteps, double *ms_out) {
    if (!h || !ms_out || nsteps < 1) return SCP_EINVAL;
    CK(cudaSetDevice(h->device));
    CK(cudaEventRecord(h->ev0, h->stream));
    int rc = scp_gpu_step(h, nsteps);
    if (rc) return rc;
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    *ms_out = ms;
    return SCP_OK;
}

void *scp_gpu_stream(scp_gpu *h) { return h ? (void *)h->stream : nullptr; }

void scp_gpu_free(scp_gpu *h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->snap_pending) cudaEventSynchronize(h->snap_done);
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
    if (h->stream) {
        void *bufs[] = {h->slab32, h->slab, h->part, h->fold, h->cg, h->point, h->flag, h->count, h->stage,
                        h->snap_dev, h->raux, h->kacc, h->dpart, h->drho};
        for (void *b : bufs)
            if (b) cudaFreeAsync(b, h->stream);
        cudaStreamSynchronize(h->stream);
    }
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->snap_ready) cudaEventDestroy(h->snap_ready);
    if (h->snap_done) cudaEventDestroy(h->snap_done);
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

const char *scp_gpu_errstr(int code) {
    switch (code) {
        case SCP_OK: return "ok";
        case SCP_EINVAL: return "invalid argument";
        case SCP_ENOMEM: return "device out of memory";
        case SCP_ECUDA: return "CUDA runtime error";
        case SCP_ENETCHARGE: return "gauged periodic seed is not net-neutral (use +/- pairs or bc_type=0)";
        case SCP_EGAUSS: return "Gauss projection did not converge";
        case SCP_ENONFINITE: return "non-finite field value";
        case SCP_EUNSUPPORTED: return "configuration not supported";
        case SCP_ENODEV: return "no CUDA device";
        case SCP_EBUSY: return "busy";
        case SCP_ETIMEOUT: return "bounded wait expired";
        default: return "unknown error";
    }
}

const char *scp_gpu_last_cuda_error(void) { return g_cuda_err; }

int scp_gpu_abi_version(void) { return SCP_GPU_ABI_VERSION; }

}  // extern "C"

__global__ void trig_check_kernel(const double *x, int n, double *err) {
    __shared__ double red[4][256];
    double e[4] = {0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s, c, rs, rc;
        sincos_bounded(x[i], &s, &c);
        sincos(x[i], &rs, &rc);
        e[0] = fmax(e[0], fabs(s - rs));
        e[1] = fmax(e[1], fabs(c - rc));
        float sf, cf, rsf, rcf;
        sincos_bounded((float)x[i], &sf, &cf);
        sincosf((float)x[i], &rsf, &rcf);
        e[2] = fmax(e[2], (double)fabsf(sf - rsf));
        e[3] = fmax(e[3], (double)fabsf(cf - rcf));
    }
    for (int q = 0; q < 4; q++) red[q][threadIdx.x] = e[q];
    __syncthreads();
    if (threadIdx.x < 4) {
        double m = 0;
        for (int t = 0; t < (int)blockDim.x; t++) m = fmax(m, red[threadIdx.x][t]);
        err[threadIdx.x] = m;
    }
}

extern "C" int scp_gpu_check_trig(int n, const double *x, double *err) {
    if (n < 1 || !x || !err) return SCP_EINVAL;
    double *dx = nullptr, *de = nullptr;
    CK(cudaMalloc(&dx, sizeof(double) * n));
    cudaError_t e = cudaMalloc(&de, sizeof(double) * 4);
    if (e == cudaSuccess) e = cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        trig_check_kernel<<<1, 256>>>(dx, n, de);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(err, de, sizeof(double) * 4, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(de);
    CK(e);
    return SCP_OK;
}

// ---------------------------------------------------------------- allocation-free diagnostics
//
// For callers that cannot allocate device memory (see scp_gpu_diag_noalloc
// in include/scp_gpu.h).  The reduction scratch is this file-scope device
// array: partial rows of the two reduction passes, the folded values and
// the point reads.  Its name in host code is only a stand-in for the symbol,
// so the device address is looked up with cudaGetSymbolAddress, with the
// device current, and passed to the kernels.

namespace {

constexpr int kStaticPartRows = kRedMaxBlocks;      // one row of 32 doubles per CTA
constexpr size_t kStaticDoubles = (size_t)kStaticPartRows * 32 + 64 + 8;
static_assert(kStaticDoubles * 8 == SCP_DIAG_STATIC_SCRATCH_BYTES, "scratch size in the header");
// red_blocks() never launches more CTAs than kRedMaxBlocks, so one partial row
// per CTA fits for every grid up to SCP_DIAG_STATIC_MAX_N per edge
static_assert(kStaticPartRows >= kRedMaxBlocks, "one partial row per reduction CTA");
static_assert(SCP_DIAG_STATIC_MAX_N <= 2048, "the static scratch limit is within the library's grid limit");

__device__ __align__(256) double g_diag_scratch[kStaticDoubles];

// Driver context current on this thread (cuCtxGetCurrent through the runtime's
// driver entry point, so the library needs no link against libcuda).
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
CUcontext current_context() {
    static CtxGetCurrentFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (CtxGetCurrentFn)f;
    }();
    CUcontext c = nullptr;
    if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
    return c;
}

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double *g_scratch_addr[kMaxDevices] = {};
CUcontext g_scratch_ctx[kMaxDevices] = {};

// Device address of g_diag_scratch for the device current on this thread.
// The lookup is made once per device and repeated only when the device's
// context has changed since (a cudaDeviceReset, or a caller that made a
// different context current), so a stale address is never handed out.
int static_scratch(int dev, double **out) {
    if (dev < 0 || dev >= kMaxDevices) return SCP_ENODEV;
    const CUcontext ctx = current_context();
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev] || !ctx || ctx != g_scratch_ctx[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_diag_scratch);
        if (e != cudaSuccess || !ptr) {
            snprintf(g_cuda_err, sizeof g_cuda_err, "cudaGetSymbolAddress(g_diag_scratch): %s",
                     cudaGetErrorString(e));
            g_scratch_addr[dev] = nullptr;
            return SCP_ECUDA;
        }
        g_scratch_addr[dev] = (double *)ptr;
        g_scratch_ctx[dev] = ctx;
    }
    *out = g_scratch_addr[dev];
    return SCP_OK;
}

// State given as the caller's 24/30 device columns in SFA order.
struct ViewCols {
    const double *pos[15];   // packed field order u v tu tv th
    const double *mom[15];   // du dv dtu dtv E
    __device__ __forceinline__ double q(int f, long long i) const { return pos[f][i]; }
    __device__ __forceinline__ double p(int f, long long i) const { return mom[f][i]; }
};

}  // namespace

extern "C" int scp_gpu_diag_noalloc(const scp_gpu_params *pp, const double *const *dev_cols, double G_offset,
                                    void *stream_ptr, scp_gpu_diag_out *out) {
    if (!pp || !dev_cols || !out) return SCP_EINVAL;
    // the size limit of the static scratch comes first, so its own message
    // reaches the caller for every grid it does not cover
    if (pp->N > SCP_DIAG_STATIC_MAX_N) {
        snprintf(g_cuda_err, sizeof g_cuda_err, "scp_gpu_diag_noalloc: N=%d exceeds SCP_DIAG_STATIC_MAX_N=%d",
                 pp->N, SCP_DIAG_STATIC_MAX_N);
        return SCP_EINVAL;
    }
    int rc = validate(pp);
    if (rc) return rc;
    if (pp->real_fields) return SCP_EUNSUPPORTED;   // takes the complex column set
    if (gext_on(pp)) return SCP_EUNSUPPORTED;        // no Higgs energy term
    if (pp->n_fabrics == 3) return SCP_EUNSUPPORTED;  // one fabric
    cudaStream_t st = (cudaStream_t)stream_ptr;
    // The call waits for its own results and copies them into a host array on
    // this stack frame, which cannot be part of a captured graph: refuse a
    // capturing stream before anything is enqueued on it.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        snprintf(g_cuda_err, sizeof g_cuda_err, "scp_gpu_diag_noalloc: the stream is capturing a graph");
        return SCP_EUNSUPPORTED;
    }
    const scp_gpu_params &p = *pp;
    const int links = p.complex_gauge ? 1 : 0;
    const int gauged = (p.complex_gauge && p.g_gauge != 0.0) ? 1 : 0;
    const int ncols = links ? 30 : 24;
    ViewCols V;
    for (int f = 0; f < 15; f++) { V.pos[f] = nullptr; V.mom[f] = nullptr; }
    for (int c = 0; c < ncols; c++) {
        if (!dev_cols[c]) return SCP_EINVAL;
        int field, mom;
        sfa_col_source(c, &field, &mom);
        (mom ? V.mom : V.pos)[field] = dev_cols[c];
    }
    if (!links)   // ungauged diagnostics never read links or E; keep the pointers valid anyway
        for (int f = FTH; f < FTH + 3; f++) { V.pos[f] = V.pos[FU]; V.mom[f] = V.mom[FU]; }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    double *scratch = nullptr;
    if ((rc = static_scratch(dev, &scratch))) return rc;
    double *part = scratch, *fold = scratch + (size_t)kStaticPartRows * 32, *point = fold + 64;
    const long long n3 = (long long)p.N * p.N * p.N;
    const int nb = red_blocks(n3);
    const DiagConsts c = diag_consts_for(p, gauged, links, 0, G_offset);
    // every scratch word read below is written first in the same call (each
    // CTA writes its whole partial row, the folds write their outputs), so
    // no clearing is needed; the fold area is zeroed only so a failed launch
    // cannot hand back the previous call's numbers
    CK(cudaMemsetAsync(fold, 0, sizeof(double) * (64 + 8), st));
    diag_pass1_kernel<ViewCols><<<nb, kRedThreads, 0, st>>>(V, c, part);
    fold_partials_kernel<DS_NSUM, DM_NMAX><<<1, 1024, 0, st>>>(part, nb, fold);
    diag_pass2_kernel<ViewCols><<<nb, kRedThreads, 0, st>>>(V, c, fold, part);
    fold_partials_kernel<1, 1><<<1, 1024, 0, st>>>(part, nb, fold + 40);
    diag_point_kernel<ViewCols><<<1, 32, 0, st>>>(V, c, fold + 41, p.qdiag_probe1, p.qdiag_probe2, point);
    CK(cudaGetLastError());
    double h[53];
    CK(cudaMemcpyAsync(h, fold, sizeof(double) * 42, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(h + 48, point, sizeof(double) * 5, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    diag_assemble(h, h + 40, h + 48, c, n3, p.g_gauge, out);
    if (!isfinite(out->v[SCP_DIAG_E_TOTAL])) return SCP_ENONFINITE;
    return SCP_OK;
}

#include "serve.cuh"
