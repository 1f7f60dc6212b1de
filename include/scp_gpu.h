/* scp_gpu.h -- C ABI of libscpgpu.so, the B200 (sm_100a) lattice time-stepper
 * for the complex / gauged Cosserat Q-ball model of kardianos/scp sfa/sim.
 *
 * The reference keeps its GPU stepper as file-static host functions inside
 * the driver translation unit (sfa/sim/scp_sim.cu).  This header replaces
 * that set with an opaque-handle C ABI: plain pointers and sizes, no CUDA or
 * C++ types, every call returns a status code and nothing calls exit().
 *
 *   reference (sfa/sim/scp_sim.cu)                 replaced by
 *   gpu_alloc            :2659  cudaMalloc per array  scp_gpu_init
 *   gpu_set_constants    :2915  __constant__ copies   scp_gpu_init
 *   gpu_upload           :2768  H2D of all columns    scp_gpu_init
 *   host init_gauss_project + first force :5151-5245  scp_gpu_init (on device)
 *   gpu_verlet_step      :2971  9-12 launches/step    scp_gpu_step (1 launch/step)
 *   run_gpu_diagnostics  :3764  atomics + D2H         scp_gpu_diag (deterministic)
 *   snap_hook/downcast   :3607, :1734                 scp_gpu_snapshot
 *   gpu_download         :2822                        scp_gpu_snapshot (dtype f64)
 *   gpu_free             :2880                        scp_gpu_free
 *
 * Column order of host_cols[] is the SFA registration order of the reference
 * snapshot writer (sfa/sim/scp_sim.c:2862-2897):
 *    0- 2 phi_x..z   3- 5 theta_x..z   6- 8 phi_vx..vz   9-11 theta_vx..vz
 *   12-14 phiim_*   15-17 thetaim_*   18-20 phiim_v*    21-23 thetaim_v*
 *   24-26 th_x..z   27-29 E_x..z      (24-29 only when complex_gauge=1)
 *   30-32 th2_x..z  33-35 E2_x..z     (snapshots only, when g_gauge2 != 0:
 *                                      the second gauge starts at zero, as the
 *                                      reference's SFA seed loader leaves it)
 * Three fabrics (n_fabrics = 3): the 30 columns above are fabric C with the
 * shared links; init takes 48 more, fabric Q (30-53) then fabric L (54-77),
 * each in the 24-column complex order 0-23; snapshots carry C and then L
 * (30-53: lphi_*, lth_*, lphi_v*, lth_v*, lphiim_*, lthim_*, lphiim_v*,
 * lthim_v*), the reference's schema (scp_sim.c:2907-2932).
 * Each column is N^3 values, site index (i*N + j)*N + k, k fastest.
 *
 * Threading: one handle is driven by one host thread at a time.  Every handle
 * owns its own CUDA stream; distinct handles may run concurrently.
 */
#ifndef SCP_GPU_H
#define SCP_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SCP_GPU_ABI_VERSION 6
#define SCP_GPU_MAX_COLS 78

/* status codes */
#define SCP_OK              0
#define SCP_EINVAL         -1   /* bad parameter or handle */
#define SCP_ENOMEM         -2   /* device allocation failed */
#define SCP_ECUDA          -3   /* CUDA runtime error (see scp_gpu_last_cuda_error) */
#define SCP_ENETCHARGE     -4   /* gauged + periodic seed is not net-neutral */
#define SCP_EGAUSS         -5   /* Gauss projection CG did not converge */
#define SCP_ENONFINITE     -6   /* a field went NaN/Inf (device flag) */
#define SCP_EUNSUPPORTED   -7   /* configuration outside the implemented subset */
#define SCP_ENODEV         -8   /* no usable CUDA device */
#define SCP_EBUSY          -9   /* serving queue full / request slot unavailable */
#define SCP_ETIMEOUT      -10   /* a bounded device wait gave up */

/* precision modes */
#define SCP_PREC_FP64   0   /* all state and arithmetic in FP64 */
#define SCP_PREC_FP32C  1   /* FP32 state, compensated hi/lo positions, FP64 reductions */

/* snapshot dtypes: the SFA dtype codes (sfa/format/sfa.h:86-90) */
#define SCP_DTYPE_F16 0
#define SCP_DTYPE_F32 1
#define SCP_DTYPE_F64 2

/* Physics / grid parameters: the subset of the reference Config that the
 * complex (complex_phi=1) and gauged (complex_gauge=1) stepper reads
 * (sfa/sim/scp_config.h:22-160).  Masses are passed squared, as the reference
 * stores them after cfg_set (scp_config.h:222-223). */
typedef struct {
    int32_t N;                /* grid edge, >= 3 */
    double  L;                /* half width; the caller passes dx = 2L/(N-1) */
    double  dx, dt;           /* dt = dt_factor*dx (scp_sim.c:204-205) */
    double  m2, mtheta2, eta, mu, kappa;
    int32_t complex_gauge;    /* 1: compact U(1) links on every link */
    double  g_gauge;          /* gauge coupling >= 0; with complex_gauge=1 and g_gauge=0 the
                                 ungauged dynamics run and th / E are carried unchanged, as
                                 the reference dispatches (scp_sim.c:1586, :2820) */
    int32_t bc_type;          /* 0 absorbing sphere, 2 periodic (1 unsupported) */
    double  damp_width, damp_rate;
    int32_t precision_mode;   /* SCP_PREC_FP64 or SCP_PREC_FP32C */
    double  qdiag_radius, qdiag_probe1, qdiag_probe2;
    int32_t gauss_project;    /* 1: one-time Gauss projection at init (reference default) */
    int32_t device;           /* CUDA device ordinal */
    int32_t tile_variant;     /* 0: autotuned default; >0 selects a fixed tile shape */
    int32_t real_fields;      /* 1: the reference's real 6-field mode (complex_phi=0,
                                 compute_forces scp_sim.c:743-929 with its default terms):
                                 12 host columns (0-11 of the order above), run as the
                                 complex dynamics with a zero imaginary sector, which is the
                                 same equation of motion; not with complex_gauge */
    /* Optional terms of the real 6-field mode (compute_forces, scp_sim.c:743-929; all
     * zero = the default terms): mass mode 1 (m_eff^2 = inv_alpha/(1+inv_beta|phi|^2))
     * or 3 (kappa_eff = kappa/(1+kappa_gamma|phi|^2)), Cosserat strain alpha_cs,
     * curl-squared hardening beta_h, chiral helicity kappa_h.  With any of them set the
     * real mode runs on its own FP64 plane-ring kernels (FP32C refused). */
    int32_t mode;
    double  inv_alpha, inv_beta, kappa_gamma, alpha_cs, beta_h, kappa_h;
    /* Extensions of the gauged stepper (complex_gauge=1 and g_gauge != 0; ignored
     * without complex_gauge, as the reference ignores them; refused with g_gauge = 0
     * and in FP32C).  Higgs condensate (higgs_v > 0): V_H = (higgs_lam/4)(H^2 - v^2)^2
     * + (higgs_kap/2) s H^2, H starting at v, or with a tanh cavity of radius
     * higgs_rvoid (scp_sim.c:2802-2817).  Second compact U(1) gauge (g_gauge2 != 0)
     * with per-component charges gauge2_q[3] (scp_config.h:97-103); its links and
     * field start at zero and are Gauss-projected at init.  Either runs on one fused
     * FP64 plane-ring kernel per step. */
    double  higgs_v, higgs_lam, higgs_kap, higgs_rvoid;
    double  g_gauge2;
    double  gauge2_q[3];
    /* Three matter fabrics C, Q, L under the shared links (n_fabrics = 3; needs
     * complex_gauge = 1 and g_gauge != 0, not with the Higgs or the second gauge;
     * FP64).  Each fabric has its own bag and couples to the links with charge
     * q_fab[f] (q_C, q_Q, q_L); the Gauss law uses sum_f q_f rho_f.  mf_lock_CQ = 1
     * keeps Q equal to C at every step (the Q columns passed to init are then
     * ignored); 0 evolves Q on its own (scp_config.h:135-149).  A step is one FP64
     * plane-ring kernel per fabric and one for the links. */
    int32_t n_fabrics;
    int32_t mf_lock_CQ;
    double  q_fab[3];
} scp_gpu_params;

/* Diagnostic slots: the reference diag TSV columns after "t"
 * (sfa/sim/scp_sim.c:2993-3003), same order and meaning. */
enum {
    SCP_DIAG_E_PHI_KIN = 0, SCP_DIAG_E_THETA_KIN, SCP_DIAG_E_GRAD, SCP_DIAG_E_MASS,
    SCP_DIAG_E_POT, SCP_DIAG_E_TGRAD, SCP_DIAG_E_TMASS, SCP_DIAG_E_COUPLING,
    SCP_DIAG_E_TOTAL, SCP_DIAG_PHI_MAX, SCP_DIAG_P_MAX, SCP_DIAG_P_INT, SCP_DIAG_THETA_RMS,
    SCP_DIAG_Q_PHI, SCP_DIAG_Q_THETA, SCP_DIAG_Q_TOTAL, SCP_DIAG_S_MAX, SCP_DIAG_R_CORE,
    SCP_DIAG_OMEGA_CORE, SCP_DIAG_Q_CORE, SCP_DIAG_THP1U, SCP_DIAG_THP1V, SCP_DIAG_THP2U,
    SCP_DIAG_THP2V, SCP_DIAG_GAUSS_MAX, SCP_DIAG_GAUSS_L2, SCP_DIAG_E_EM, SCP_DIAG_Q_FLUX,
    SCP_DIAG_Q_P0, SCP_DIAG_Q_P1, SCP_DIAG_Q_P2,
    SCP_DIAG_CENTROID_X, SCP_DIAG_CENTROID_Y, SCP_DIAG_CENTROID_Z,
    /* three fabrics only (compute_mf_charges, scp_sim.c:2247-2261): integrated
     * Noether charge of C, Q, L and the EM charge sum_f q_f Q_f */
    SCP_DIAG_Q_C, SCP_DIAG_Q_Q, SCP_DIAG_Q_L, SCP_DIAG_Q_EM,
    SCP_DIAG_NSLOTS = 40
};
typedef struct { double v[SCP_DIAG_NSLOTS]; } scp_gpu_diag_out;

typedef struct {
    int64_t steps_done;       /* leapfrog steps taken since init */
    double  time;             /* steps_done * dt */
    double  G_offset;         /* frozen Gauss offset measured after projection */
    int32_t cg_iterations;    /* Gauss projection CG iterations after the spectral start
                                 (the direct FFT solve of the same periodic 7-point problem,
                                 for power-of-two N up to 512 and other N up to 192): 0 when
                                 the start already meets the reference's stopping rule */
    int32_t precision_mode;
    int64_t device_bytes;     /* device memory held by the handle */
    double  state_bytes_per_site;   /* persistent bytes per site of the layout */
    double  step_bytes_per_site;    /* algorithmic bytes moved per site-update */
    int32_t tile_x, tile_y, seg_len; /* tile shape in use */
    int32_t sites_per_thread; /* 2: two-site packed FP32C kernel (even N), else 1 */
    int32_t tma_staging;      /* form of the FP64 step: 0 the cp.async ring (the default); on
                                 full tiles of the default shapes SCP_STAGING=tma in the
                                 environment selects TMA tile loads of the positions (1) and
                                 SCP_STAGING=cpm the cp.async ring with TMA-staged momenta (2),
                                 both bit-identical to 0; on gauged grids with the default tile
                                 SCP_STAGING=duo selects two threads per site (3, equal to 0 up
                                 to roundoff) */
} scp_gpu_info;

typedef struct scp_gpu scp_gpu;

/* Allocate device state, upload the host columns (12 real, 24 complex, 30 gauged,
 * 78 with three fabrics),
 * and run the start-up sequence of the reference main (scp_sim.cu:5151-5245):
 * net-charge check (gauged, periodic), Gauss projection, first force. */
int  scp_gpu_init(const scp_gpu_params *p, const double *const *host_cols, scp_gpu **out);
/* Same as scp_gpu_init, but the columns are device pointers (no H2D copy). */
int  scp_gpu_init_device(const scp_gpu_params *p, const double *const *dev_cols, scp_gpu **out);
/* Enqueue nsteps fused leapfrog steps on the handle's stream (asynchronous). */
int  scp_gpu_step(scp_gpu *h, int nsteps);
/* Wait for all work on the handle's stream; reports a pending NaN/Inf flag. */
int  scp_gpu_sync(scp_gpu *h);
/* FP64 reductions of the current state; synchronises.  Deterministic. */
int  scp_gpu_diag(scp_gpu *h, scp_gpu_diag_out *out);
/* Copy the current state to host columns in dtype (SCP_DTYPE_*); the f32/f16
 * casts are done on the device with the reference's conversion rules. */
int  scp_gpu_snapshot(scp_gpu *h, int dtype, void *const *host_cols);
/* Asynchronous snapshot, the overlapped form of the reference's snap_hook
 * (scp_sim.cu:3496-3691: down-cast kernels, pinned buffers, async D2H).  The
 * down-conversion into device staging runs on the handle's stream, so steps
 * enqueued after this call see it finished before they overwrite the state;
 * the copies into host_cols run on a separate copy stream and overlap with
 * those steps.  host_cols must stay valid until scp_gpu_snapshot_wait
 * returns (page-locked memory from scp_gpu_host_alloc makes the copies truly
 * asynchronous).  One snapshot is in flight per handle: a second call first
 * waits for the previous one.  The staging (ncols x N^3 x dtype size) is
 * allocated on first use and kept until scp_gpu_free. */
int  scp_gpu_snapshot_async(scp_gpu *h, int dtype, void *const *host_cols);
/* Wait until the snapshot in flight (if any) has landed in host memory. */
int  scp_gpu_snapshot_wait(scp_gpu *h);
/* Page-locked host memory for snapshot buffers (NULL on failure). */
void *scp_gpu_host_alloc(size_t bytes);
void scp_gpu_host_free(void *p);
int  scp_gpu_get_info(const scp_gpu *h, scp_gpu_info *info);
/* Time nsteps on the handle's stream with CUDA events recorded on that
 * stream; *ms_out receives the device time of the whole batch. */
int  scp_gpu_time_steps(scp_gpu *h, int nsteps, double *ms_out);
/* The handle's cudaStream_t, as an opaque pointer. */
void *scp_gpu_stream(scp_gpu *h);
void scp_gpu_free(scp_gpu *h);
const char *scp_gpu_errstr(int code);
const char *scp_gpu_last_cuda_error(void);
int  scp_gpu_abi_version(void);
/* Self-check of the library's bounded-argument sine/cosine (used by the
 * gauged step in place of the CUDA math library) against CUDA's sin/cos on
 * device: for the n host angles x[], err[0..3] receive the largest absolute
 * difference of sin and cos in FP64 and of sin and cos in FP32.  Synchronous;
 * allocates and frees its own device buffers. */
int  scp_gpu_check_trig(int n, const double *x, double *err);

/* Diagnostics for callers that must not allocate device memory.
 *
 * No counterpart in the reference.  Some hosts of this library cannot call
 * cudaMalloc while they run a simulation: a process whose device memory is
 * carved up and owned by another framework (its allocator holds the whole
 * pool, so a cudaMalloc outside it fails or fragments that pool), or a
 * real-time loop that treats any allocation, with its implicit device
 * synchronisation, as a failure.  This entry point computes the same
 * diagnostics as scp_gpu_diag for a state that the caller already holds on
 * the device, without a handle and without allocating: its reduction scratch
 * is a fixed array that lives in the library (SCP_DIAG_STATIC_SCRATCH_BYTES,
 * about 300 KB, held by every GPU that loads the library until the process
 * exits).
 *
 *   p          grid and physics parameters (as for scp_gpu_init)
 *   dev_cols   24 or 30 device pointers, FP64 columns in the SFA order above
 *   G_offset   frozen Gauss offset to measure against (scp_gpu_info.G_offset)
 *   stream     cudaStream_t to run on, or NULL for the legacy default stream
 *   out        host result, slot order as scp_gpu_diag
 *
 * Grids larger than SCP_DIAG_STATIC_MAX_N per edge are rejected with
 * SCP_EINVAL (scp_gpu_last_cuda_error names the limit).  The first call on
 * a device (and the first after that device's context changed, e.g. after
 * cudaDeviceReset) looks up the scratch array's device address; the call
 * waits on `stream` and reads its results into host memory, so it must be
 * made outside stream capture: on a capturing stream it returns
 * SCP_EUNSUPPORTED before enqueuing anything.  All calls share the one
 * scratch array, so calls whose work overlaps on the GPU (two host threads,
 * or two streams) race: serialise them.  The call synchronises on `stream`
 * before it returns. */
#define SCP_DIAG_STATIC_MAX_N 2048
#define SCP_DIAG_STATIC_SCRATCH_BYTES (8 * (1184 * 32 + 64 + 8))
int  scp_gpu_diag_noalloc(const scp_gpu_params *p, const double *const *dev_cols, double G_offset,
                          void *stream, scp_gpu_diag_out *out);

/* ------------------------------------------------------------------ serving
 *
 * Continuous-batching server for many independent simulations on one GPU
 * (no counterpart in the reference, which runs one simulation per process).
 * Requests of any grid size are queued by scp_srv_submit, admitted by
 * scp_srv_poll while active slots (max_active) and the HBM budget allow,
 * and advanced together: every poll runs one chunk of chunk_steps steps in
 * which one persistent launch per step advances every active request,
 * replayed as a captured CUDA graph.  Requests that arrive while others run
 * join at the next chunk boundary; a finished request is retired at the end
 * of its chunk (final diagnostics, optional snapshot into the caller's
 * out_cols, device memory freed).  The tile shape of each (grid size, gauge
 * mode, precision) is picked by timing every compiled shape once (autotune).
 * A request's state evolves exactly as it would through scp_gpu_step. */
typedef struct scp_srv scp_srv;

typedef struct {
    int32_t device;
    int32_t max_active;        /* concurrently admitted requests (<= 256 per group) */
    int64_t mem_budget_bytes;  /* device bytes for admitted state; 0 = unlimited */
    int32_t chunk_steps;       /* steps per poll (graph length) */
    int32_t use_graph;         /* 1: replay chunks as a CUDA graph */
    int32_t autotune;          /* 1: time the tile shapes per grid size */
    int32_t admit_per_poll;    /* loaded requests taken into the active set per poll
                                  (0 = no cap) */
    int32_t loader_threads;    /* threads initialising queued requests (upload, Gauss
                                  projection) while chunks run; 0 = 4.  Their work runs on
                                  high-priority streams so it interleaves with the chunks. */
} scp_srv_config;

#define SCP_SRV_QUEUED 0
#define SCP_SRV_ACTIVE 1
#define SCP_SRV_DONE   2
#define SCP_SRV_FAILED 3

typedef struct {
    int32_t state, rc;
    double  t_submit, t_admit, t_done;   /* host monotonic seconds */
    int64_t nsteps;
    int32_t N, tile_variant;
} scp_srv_request_info;

typedef struct {
    int64_t step, chunks, mem_in_use;
    int32_t n_active, n_queued, n_groups;
    double  t_admit, t_autotune, t_run, t_retire;   /* host seconds spent per phase; t_admit and
                                                       t_autotune are summed over the loader
                                                       threads, t_retire over the two retire
                                                       threads (final step, diagnostics, free) */
    double  t_wait;           /* poll time spent waiting for a first loaded request */
    double  t_launch;         /* poll time spent planning, uploading tables, launching */
    double  t_gpu;            /* device time of the chunks (CUDA events on the server stream) */
} scp_srv_stats_t;

int  scp_srv_create(const scp_srv_config *cfg, scp_srv **out);
/* Queue a request.  The columns are copied, so host_cols may be released on
 * return; scp_srv_submit_borrowed instead keeps the pointers, which must stay
 * valid until the request is admitted (state no longer SCP_SRV_QUEUED).
 * out_cols (optional, NULL for none) receive the final snapshot in out_dtype
 * and must stay valid until the request is done. */
int  scp_srv_submit(scp_srv *s, const scp_gpu_params *p, const double *const *host_cols, int64_t nsteps,
                    void *const *out_cols, int out_dtype, int64_t *id_out);
int  scp_srv_submit_borrowed(scp_srv *s, const scp_gpu_params *p, const double *const *host_cols, int64_t nsteps,
                             void *const *out_cols, int out_dtype, int64_t *id_out);
/* Take in the requests the loader threads have initialised, finish the chunk
 * in flight, launch the next one, hand finished requests to the retire
 * threads; reports the active count (running or retiring) and the queued
 * count (queued, loading or loaded but not yet taken). */
int  scp_srv_poll(scp_srv *s, int *n_active, int *n_queued);
int  scp_srv_status(scp_srv *s, int64_t id, scp_srv_request_info *info);
/* Final diagnostics of a finished request (SCP_EBUSY while queued/active). */
int  scp_srv_result(scp_srv *s, int64_t id, scp_gpu_diag_out *diag);
int  scp_srv_stats(scp_srv *s, scp_srv_stats_t *st);
void scp_srv_free(scp_srv *s);

#ifdef __cplusplus
}
#endif
#endif /* SCP_GPU_H */
