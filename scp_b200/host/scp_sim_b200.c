/* scp_sim_b200.c -- config-driven host driver for the B200 stepper.
 *
 * The reference runs its complex / gauged simulations through `main` in
 * sfa/sim/scp_sim.c (CPU) and sfa/sim/scp_sim.cu (CUDA): read a key = value
 * config or resume from an .sfa file's KVMD, initialise the fields, write SFA
 * snapshots and a diagnostic TSV while stepping.  This driver keeps that flow
 * and those files -- it compiles the reference's own scp_config.h (Config,
 * parser, validation), scp_init.h (initial states, KVMD embedding) and
 * sfa/format/sfa.h (the archive) -- and replaces the stepper with the C ABI of
 * libscpgpu.so (include/scp_gpu.h).
 *
 *   scp_sim_b200 config.cfg [-key value ...]
 *   scp_sim_b200 run.sfa    [-key value ...]      resume from the last frame
 *
 * Extra keys read by this driver only (not passed to the reference parser):
 *   gpu_precision  = fp64 | fp32c   (default fp64)
 *   gpu_device     = <ordinal>       (default 0)
 *   gpu_async_snap = 1 | 0          (default 1: snapshots copied and written
 *                                     while the GPU keeps stepping)
 * It covers the complex (complex_phi=1), gauged (complex_gauge=1, with the
 * Higgs condensate, the second gauge or three matter fabrics) and real
 * 6-field (complex_phi=0, with its optional terms) stepper with bc_type 0 or
 * 2; other modes are refused with a message.
 *
 * Build: make -C scp_b200/host REF=<kardianos/scp checkout>
 */
#define SFA_IMPLEMENTATION
#include "sfa.h"
#include "scp_config.h"

#include <pthread.h>
#include <stdint.h>
#include <time.h>

#include "scp_gpu.h"

/* Host staging grid with the members scp_init.h reads (sfa/sim/scp_init.h:1-8). */
typedef struct {
    double *mem;
    double *phi[3], *phi_vel[3], *theta[3], *theta_vel[3];
    double *phi_im[3], *phi_im_vel[3], *theta_im[3], *theta_im_vel[3];
    double *th[3], *Efield[3];
    int N;
    long N3;
    double L, dx, dt;
} Grid;

#define SCP_COMPLEX_FIELDS 1
#include "scp_init.h"

static double wall_now(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* Host arrays in SFA column order (24 or 30 columns of N^3 doubles; 78 with
 * three fabrics: C, Q, L). */
static Grid *grid_new(const Config *c, double **cols, int ncols) {
    Grid *g = calloc(1, sizeof(Grid));
    if (!g) return NULL;
    g->N = c->N;
    g->N3 = (long)c->N * c->N * c->N;
    g->L = c->L;
    g->dx = 2.0 * c->L / (c->N - 1);
    g->dt = c->dt_factor * g->dx;
    g->mem = calloc((size_t)ncols * g->N3, sizeof(double));
    if (!g->mem) { free(g); return NULL; }
    for (int k = 0; k < ncols; k++) cols[k] = g->mem + (size_t)k * g->N3;
    for (int a = 0; a < 3; a++) {
        g->phi[a] = cols[0 + a];      g->theta[a] = cols[3 + a];
        g->phi_vel[a] = cols[6 + a];  g->theta_vel[a] = cols[9 + a];
        g->phi_im[a] = cols[12 + a];  g->theta_im[a] = cols[15 + a];
        g->phi_im_vel[a] = cols[18 + a]; g->theta_im_vel[a] = cols[21 + a];
        g->th[a] = ncols >= 30 ? cols[24 + a] : NULL;
        g->Efield[a] = ncols >= 30 ? cols[27 + a] : NULL;
    }
    return g;
}

/* Fabric L's snapshot columns (scp_sim.c:2907-2932): names, and semantic /
 * component as fabric C's complex columns 0-23. */
static const char *l_names[24] = {
    "lphi_x", "lphi_y", "lphi_z", "lth_x", "lth_y", "lth_z",
    "lphi_vx", "lphi_vy", "lphi_vz", "lth_vx", "lth_vy", "lth_vz",
    "lphiim_x", "lphiim_y", "lphiim_z", "lthim_x", "lthim_y", "lthim_z",
    "lphiim_vx", "lphiim_vy", "lphiim_vz", "lthim_vx", "lthim_vy", "lthim_vz"};

/* Column schema of the complex / gauged snapshot (sfa/sim/scp_sim.c:2862-2932;
 * th2 / E2 with the second gauge; fabric L after C with three fabrics). */
static void add_columns(SFA *sfa, uint8_t dt, int n, int fabrics) {
    static const char *names[36] = {
        "phi_x", "phi_y", "phi_z", "theta_x", "theta_y", "theta_z",
        "phi_vx", "phi_vy", "phi_vz", "theta_vx", "theta_vy", "theta_vz",
        "phiim_x", "phiim_y", "phiim_z", "thetaim_x", "thetaim_y", "thetaim_z",
        "phiim_vx", "phiim_vy", "phiim_vz", "thetaim_vx", "thetaim_vy", "thetaim_vz",
        "th_x", "th_y", "th_z", "E_x", "E_y", "E_z",
        "th2_x", "th2_y", "th2_z", "E2_x", "E2_y", "E2_z"};
    static const uint8_t sem[36] = {
        SFA_POSITION, SFA_POSITION, SFA_POSITION, SFA_ANGLE, SFA_ANGLE, SFA_ANGLE,
        SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY,
        SFA_POSITION, SFA_POSITION, SFA_POSITION, SFA_ANGLE, SFA_ANGLE, SFA_ANGLE,
        SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY,
        SFA_ANGLE, SFA_ANGLE, SFA_ANGLE, SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY,
        SFA_ANGLE, SFA_ANGLE, SFA_ANGLE, SFA_VELOCITY, SFA_VELOCITY, SFA_VELOCITY};
    static const uint8_t comp[36] = {0, 1, 2, 0, 1, 2, 0, 1, 2, 3, 4, 5, 3, 4, 5, 3, 4, 5,
                                     6, 7, 8, 9, 10, 11, 6, 7, 8, 12, 13, 14, 9, 10, 11, 15, 16, 17};
    if (fabrics == 3) {
        for (int k = 0; k < 30; k++) sfa_add_column(sfa, names[k], dt, sem[k], comp[k]);
        for (int k = 0; k < 24; k++) sfa_add_column(sfa, l_names[k], dt, sem[k], comp[k]);
        return;
    }
    for (int k = 0; k < n; k++) sfa_add_column(sfa, names[k], dt, sem[k], comp[k]);
}

/* One fabric from an SFA frame into 24 complex columns, each source column
 * placed by its semantic and component as load_sfa_into_fabric does
 * (scp_sim.c:426-479; gauge columns are not loaded). */
static int load_fabric(const char *path, int frame, int N, double **cols24) {
    SFA *sfa = sfa_open(path);
    if (!sfa) { fprintf(stderr, "FATAL: cannot open SFA '%s'\n", path); return 1; }
    if ((int)sfa->Nx != N || (int)sfa->Ny != N || (int)sfa->Nz != N) {
        fprintf(stderr, "FATAL: SFA grid %ux%ux%u != sim %d^3\n", sfa->Nx, sfa->Ny, sfa->Nz, N);
        sfa_close(sfa);
        return 1;
    }
    if (frame < 0) frame = (int)sfa->total_frames + frame;
    if (frame < 0 || frame >= (int)sfa->total_frames) {
        fprintf(stderr, "FATAL: frame %d out of range [0,%u)\n", frame, sfa->total_frames);
        sfa_close(sfa);
        return 1;
    }
    uint8_t *buf = malloc(sfa->frame_bytes);
    if (!buf) { sfa_close(sfa); return 1; }
    sfa_read_frame(sfa, frame, buf);
    const long n3 = (long)N * N * N;
    uint64_t off = 0;
    int nload = 0;
    for (uint32_t col = 0; col < sfa->n_columns; col++) {
        const int dtype = sfa->columns[col].dtype, sem = sfa->columns[col].semantic;
        const int comp = sfa->columns[col].component;
        const uint8_t *src = buf + off;
        int slot = -1;   /* index into the complex 24-column order */
        if (sem == SFA_POSITION && comp < 3) slot = comp;
        else if (sem == SFA_ANGLE && comp < 3) slot = 3 + comp;
        else if (sem == SFA_VELOCITY && comp < 3) slot = 6 + comp;
        else if (sem == SFA_VELOCITY && comp < 6) slot = 9 + comp - 3;
        else if (sem == SFA_POSITION && comp < 6) slot = 12 + comp - 3;
        else if (sem == SFA_ANGLE && comp < 6) slot = 15 + comp - 3;
        else if (sem == SFA_VELOCITY && comp < 9) slot = 18 + comp - 6;
        else if (sem == SFA_VELOCITY && comp < 12) slot = 21 + comp - 9;
        if (slot >= 0) {
            double *dst = cols24[slot];
            for (long i = 0; i < n3; i++)
                dst[i] = dtype == SFA_F64 ? ((const double *)src)[i]
                       : dtype == SFA_F32 ? (double)((const float *)src)[i]
                                          : f16_to_f64(((const uint16_t *)src)[i]);
            nload++;
        }
        off += (uint64_t)n3 * sfa_dtype_size[dtype];
    }
    printf("  Loaded %d columns into fabric from %s\n", nload, path);
    free(buf);
    sfa_close(sfa);
    return 0;
}

/* Snapshot pipeline: two host buffer sets (page-locked when available).
 * snap_start begins a device snapshot into a free set (down-conversion on the
 * stepping stream, copy on the library's copy stream); snap_flush, called
 * right after the next steps are enqueued, waits for the copy and queues the
 * set to a writer thread that compresses and appends the frame
 * (sfa_write_frame) while the GPU keeps stepping.  With async = 0 every frame
 * is taken and written synchronously, as the reference's CPU path does. */
typedef struct {
    scp_gpu *h;
    SFA *sfa;
    int ncols, dtype, async;
    size_t col_bytes;
    void *cols[2][54];
    int pinned[2];
    double t[2];
    int busy[2];          /* set queued to or being written by the writer */
    int queue[2], qn;     /* FIFO of sets to write */
    int next, pending;    /* next set to fill; set whose copy is in flight (-1 none) */
    int stop, werr;
    pthread_t thr;
    pthread_mutex_t mu;
    pthread_cond_t cv;
} Snap;

static void *snap_writer(void *arg) {
    Snap *s = arg;
    pthread_mutex_lock(&s->mu);
    for (;;) {
        while (!s->stop && s->qn == 0) pthread_cond_wait(&s->cv, &s->mu);
        if (s->qn == 0) break;
        const int k = s->queue[0];
        s->queue[0] = s->queue[1];
        s->qn--;
        pthread_mutex_unlock(&s->mu);
        sfa_write_frame(s->sfa, s->t[k], s->cols[k]);
        pthread_mutex_lock(&s->mu);
        s->busy[k] = 0;
        pthread_cond_broadcast(&s->cv);
    }
    pthread_mutex_unlock(&s->mu);
    return NULL;
}

static int snap_open(Snap *s, scp_gpu *h, SFA *sfa, int ncols, int precision, long n3, int async) {
    memset(s, 0, sizeof *s);
    s->h = h; s->sfa = sfa; s->ncols = ncols; s->async = async;
    s->dtype = precision == 0 ? SCP_DTYPE_F16 : (precision == 1 ? SCP_DTYPE_F32 : SCP_DTYPE_F64);
    s->col_bytes = (size_t)(precision == 0 ? 2 : (precision == 1 ? 4 : 8)) * (size_t)n3;
    s->pending = -1;
    for (int b = 0; b < (async ? 2 : 1); b++) {
        void *blk = async ? scp_gpu_host_alloc(s->col_bytes * ncols) : NULL;
        s->pinned[b] = blk != NULL;
        if (!blk) blk = malloc(s->col_bytes * ncols);
        if (!blk) return -1;
        for (int k = 0; k < ncols; k++) s->cols[b][k] = (char *)blk + (size_t)k * s->col_bytes;
    }
    pthread_mutex_init(&s->mu, NULL);
    pthread_cond_init(&s->cv, NULL);
    if (async && pthread_create(&s->thr, NULL, snap_writer, s)) return -1;
    return 0;
}

/* hand the frame whose copy is in flight to the writer */
static int snap_flush(Snap *s) {
    if (s->pending < 0) return 0;
    int rc = scp_gpu_snapshot_wait(s->h);
    if (rc) return rc;
    pthread_mutex_lock(&s->mu);
    s->queue[s->qn++] = s->pending;
    s->pending = -1;
    pthread_cond_broadcast(&s->cv);
    pthread_mutex_unlock(&s->mu);
    return 0;
}

static int snap_start(Snap *s, double t) {
    if (!s->async) {
        int rc = scp_gpu_snapshot(s->h, s->dtype, s->cols[0]);
        if (rc) return rc;
        sfa_write_frame(s->sfa, t, s->cols[0]);
        return 0;
    }
    int rc = snap_flush(s);
    if (rc) return rc;
    const int k = s->next;
    pthread_mutex_lock(&s->mu);
    while (s->busy[k]) pthread_cond_wait(&s->cv, &s->mu);
    s->busy[k] = 1;
    pthread_mutex_unlock(&s->mu);
    s->t[k] = t;
    if ((rc = scp_gpu_snapshot_async(s->h, s->dtype, s->cols[k]))) return rc;
    s->pending = k;
    s->next ^= 1;
    return 0;
}

/* flush the last frame, stop the writer, release the buffers */
static int snap_close(Snap *s) {
    int rc = 0;
    if (s->async) {
        rc = snap_flush(s);
        pthread_mutex_lock(&s->mu);
        s->stop = 1;
        pthread_cond_broadcast(&s->cv);
        pthread_mutex_unlock(&s->mu);
        pthread_join(s->thr, NULL);
    }
    for (int b = 0; b < (s->async ? 2 : 1); b++) {
        if (s->pinned[b]) scp_gpu_host_free(s->cols[b][0]);
        else free(s->cols[b][0]);
    }
    return rc;
}

/* One diag TSV row in the reference's column set and formats
 * (sfa/sim/scp_sim.c:2993-3003, :3045-3066). */
static void diag_row(FILE *fp, double t, const scp_gpu_diag_out *d, int gauged, int complex, int mf) {
    const double *v = d->v;
    fprintf(fp, "%.2f\t%.6e\t%.6e\t%.6e\t%.6e\t%.6e\t%.6e\t%.6e\t%.6e\t%.6e\t%.6e\t%.6e\t%.6e\t%.6e", t,
            v[SCP_DIAG_E_PHI_KIN], v[SCP_DIAG_E_THETA_KIN], v[SCP_DIAG_E_GRAD], v[SCP_DIAG_E_MASS],
            v[SCP_DIAG_E_POT], v[SCP_DIAG_E_TGRAD], v[SCP_DIAG_E_TMASS], v[SCP_DIAG_E_COUPLING],
            v[SCP_DIAG_E_TOTAL], v[SCP_DIAG_PHI_MAX], v[SCP_DIAG_P_MAX], v[SCP_DIAG_P_INT], v[SCP_DIAG_THETA_RMS]);
    if (!complex) {   /* real 6-field mode: energies and amplitudes only */
        fprintf(fp, "\n");
        return;
    }
    fprintf(fp, "\t%.12e\t%.12e\t%.12e\t%.6e\t%.6e\t%.12e\t%.12e\t%.6e\t%.6e\t%.6e\t%.6e",
            v[SCP_DIAG_Q_PHI], v[SCP_DIAG_Q_THETA], v[SCP_DIAG_Q_TOTAL], v[SCP_DIAG_S_MAX], v[SCP_DIAG_R_CORE],
            v[SCP_DIAG_OMEGA_CORE], v[SCP_DIAG_Q_CORE], v[SCP_DIAG_THP1U], v[SCP_DIAG_THP1V], v[SCP_DIAG_THP2U],
            v[SCP_DIAG_THP2V]);
    if (gauged)
        fprintf(fp, "\t%.6e\t%.6e\t%.12e\t%.12e", v[SCP_DIAG_GAUSS_MAX], v[SCP_DIAG_GAUSS_L2], v[SCP_DIAG_E_EM],
                v[SCP_DIAG_Q_FLUX]);
    if (mf)
        fprintf(fp, "\t%.12e\t%.12e\t%.12e\t%.12e", v[SCP_DIAG_Q_C], v[SCP_DIAG_Q_Q], v[SCP_DIAG_Q_L],
                v[SCP_DIAG_Q_EM]);
    fprintf(fp, "\t%.12e\t%.12e\t%.12e\n", v[SCP_DIAG_Q_P0], v[SCP_DIAG_Q_P1], v[SCP_DIAG_Q_P2]);
}

static int fail(const char *what, int rc) {
    fprintf(stderr, "FATAL: %s: %s (%d) %s\n", what, scp_gpu_errstr(rc), rc, scp_gpu_last_cuda_error());
    return 1;
}

int main(int argc, char **argv) {
    Config c = cfg_defaults();
    if (argc < 2) {
        fprintf(stderr, "Usage: %s config.cfg [-key value ...]\n", argv[0]);
        fprintf(stderr, "       %s input.sfa [-key value ...]   (restart from SFA)\n", argv[0]);
        return 1;
    }
    const char *arg1 = argv[1];
    const size_t len1 = strlen(arg1);
    if (len1 > 4 && !strcmp(arg1 + len1 - 4, ".sfa")) {
        /* restart: KVMD set covering all frames as the base config, grid from the header */
        SFA *in = sfa_open(arg1);
        if (!in) { fprintf(stderr, "Cannot open SFA: %s\n", arg1); return 1; }
        static SFA_KVMDSet kv[SFA_MAX_KVMD_SETS];
        const int n_kv = sfa_read_kvmd(in, kv, SFA_MAX_KVMD_SETS);
        if (n_kv > 0) {
            SFA_KVMDSet *use = &kv[0];
            for (int i = 0; i < n_kv; i++)
                if (kv[i].first_frame == 0xFFFFFFFF) { use = &kv[i]; break; }
            for (int i = 0; i < use->n_pairs; i++) cfg_set(&c, use->keys[i], use->values[i]);
        }
        char tmp[64];
        snprintf(tmp, sizeof tmp, "%u", in->Nx); cfg_set(&c, "N", tmp);
        snprintf(tmp, sizeof tmp, "%.6f", in->Lx); cfg_set(&c, "L", tmp);
        cfg_set(&c, "init", "sfa");
        strncpy(c.init_sfa, arg1, sizeof c.init_sfa - 1);
        c.init_frame = -1;
        sfa_close(in);
    } else {
        cfg_load(&c, arg1);
    }
    int gpu_prec = SCP_PREC_FP64, gpu_dev = 0, gpu_async_snap = 1;
    for (int i = 2; i + 1 < argc; i += 2) {
        const char *key = argv[i][0] == '-' ? argv[i] + 1 : argv[i];
        if (!strcmp(key, "gpu_precision")) gpu_prec = !strcmp(argv[i + 1], "fp32c") ? SCP_PREC_FP32C : SCP_PREC_FP64;
        else if (!strcmp(key, "gpu_device")) gpu_dev = atoi(argv[i + 1]);
        else if (!strcmp(key, "gpu_async_snap")) gpu_async_snap = atoi(argv[i + 1]);
        else cfg_set(&c, key, argv[i + 1]);
    }
    cfg_print(&c);
    cfg_validate(&c);
    if (!c.complex_phi && c.complex_gauge) {
        fprintf(stderr, "ERROR: the gauge links need the complex fields (complex_phi=1)\n");
        return 1;
    }
    if (c.bc_type == 1) { fprintf(stderr, "ERROR: bc_type=1 is not supported by scp_sim_b200\n"); return 1; }
    if (c.n_locks > 0 || c.test_gauge_xform) {
        fprintf(stderr, "ERROR: locks and test_gauge_xform are not supported\n");
        return 1;
    }
    const int mf = c.n_fabrics == 3;
    if (mf && c.g_gauge == 0.0) {
        fprintf(stderr, "ERROR: n_fabrics=3 needs g_gauge != 0\n");
        return 1;
    }
    /* Higgs and second gauge: ignored without complex_gauge, as the reference does
     * (scp_sim.c:229-238); with g_gauge = 0 the reference's ungauged dispatch never
     * evolves them, which this driver refuses */
    const int gext = c.complex_gauge && (c.higgs_v > 0 || c.g_gauge2 != 0);
    if (gext && c.g_gauge == 0.0) {
        fprintf(stderr, "ERROR: higgs_v / g_gauge2 need g_gauge != 0\n");
        return 1;
    }
    if (c.bc_type == 2) { c.damp_width = 0.0; c.damp_rate = 0.0; }   /* as the CUDA reference (scp_sim.cu:5170-5172) */
    const int gauged = c.complex_gauge && c.g_gauge != 0.0;
    const int ncols = c.complex_gauge ? 30 : (c.complex_phi ? 24 : 12);
    const int snap_cols = mf ? 54 : ncols + ((c.complex_gauge && c.g_gauge2 != 0) ? 6 : 0);   /* + L or th2, E2 */
    double *cols[78] = {0};
    Grid *g = grid_new(&c, cols, mf ? 78 : ncols);   /* three fabrics: C, then Q and L (24 each) */
    if (!g) { fprintf(stderr, "FATAL: host allocation\n"); return 1; }
    printf("dx=%.4f dt=%.6f device=%d precision=%s\n\n", g->dx, g->dt, gpu_dev,
           gpu_prec == SCP_PREC_FP32C ? "fp32c" : "fp64");
    do_init(g, &c);
    if (mf) {   /* mf_post_init (scp_sim.c:485-509): L seed, then Q by lock / seed / copy / zero */
        if (c.init_sfa_L[0]) {
            if (load_fabric(c.init_sfa_L, c.init_frame, c.N, cols + 54)) return 1;
        } else {
            printf("WARNING: n_fabrics=3 but init_sfa_L empty — L fabric is zero\n");
        }
        if (c.mf_lock_CQ) {
            printf("Multi-fab: Q ← C lock (Q is C on the device)\n");
        } else if (c.init_sfa_Q[0]) {
            if (load_fabric(c.init_sfa_Q, c.init_frame, c.N, cols + 30)) return 1;
        } else if (c.mf_seed_Q) {
            for (int k = 0; k < 24; k++) memcpy(cols[30 + k], cols[k], sizeof(double) * g->N3);
        }
    }

    scp_gpu_params p;
    memset(&p, 0, sizeof p);
    p.N = c.N; p.L = c.L; p.dx = g->dx; p.dt = g->dt;
    p.m2 = c.m2; p.mtheta2 = c.mtheta2; p.eta = c.eta; p.mu = c.mu; p.kappa = c.kappa;
    p.complex_gauge = c.complex_gauge; p.g_gauge = c.g_gauge;   /* g_gauge = 0: ungauged dynamics, links carried */
    p.bc_type = c.bc_type; p.damp_width = c.damp_width; p.damp_rate = c.damp_rate;
    p.precision_mode = gpu_prec;
    p.qdiag_radius = c.qdiag_radius; p.qdiag_probe1 = c.qdiag_probe1; p.qdiag_probe2 = c.qdiag_probe2;
    p.gauss_project = 1; p.device = gpu_dev; p.tile_variant = 0;
    p.real_fields = c.complex_phi ? 0 : 1;
    p.mode = c.mode; p.inv_alpha = c.inv_alpha; p.inv_beta = c.inv_beta; p.kappa_gamma = c.kappa_gamma;
    p.alpha_cs = c.alpha_cs; p.beta_h = c.beta_h; p.kappa_h = c.kappa_h;
    p.higgs_v = c.higgs_v; p.higgs_lam = c.higgs_lam; p.higgs_kap = c.higgs_kap; p.higgs_rvoid = c.higgs_rvoid;
    p.g_gauge2 = c.g_gauge2;
    p.gauge2_q[0] = c.gauge2_q0; p.gauge2_q[1] = c.gauge2_q1; p.gauge2_q[2] = c.gauge2_q2;
    p.n_fabrics = c.n_fabrics; p.mf_lock_CQ = c.mf_lock_CQ;
    p.q_fab[0] = c.q_C; p.q_fab[1] = c.q_Q; p.q_fab[2] = c.q_L;
    scp_gpu *h = NULL;
    int rc = scp_gpu_init(&p, (const double *const *)cols, &h);
    if (rc) return fail("scp_gpu_init", rc);
    free(g->mem);
    g->mem = NULL;
    if (gauged) {
        scp_gpu_info inf;
        scp_gpu_get_info(h, &inf);
        printf("Gauss projection: %d CG iters (offset %.3e)\n", inf.cg_iterations, inf.G_offset);
    }

    const uint8_t sdt = (c.precision == 0) ? SFA_F16 : (c.precision == 1) ? SFA_F32 : SFA_F64;
    SFA *sfa = sfa_create(c.output, c.N, c.N, c.N, c.L, c.L, c.L, g->dt);
    if (!sfa) { fprintf(stderr, "ERROR: cannot create output file '%s'\n", c.output); return 1; }
    sfa->flags = SFA_CODEC_COLZSTD | SFA_FLAG_STREAMING;
    sfa_embed_kvmd(sfa, &c);
    add_columns(sfa, sdt, snap_cols, c.n_fabrics);
    sfa_finalize_header(sfa);
    static Snap snap;
    if (snap_open(&snap, h, sfa, snap_cols, c.precision, g->N3, gpu_async_snap)) {
        fprintf(stderr, "FATAL: snapshot buffers\n");
        return 1;
    }
    if ((rc = snap_start(&snap, 0.0))) return fail("snapshot", rc);

    FILE *fp = fopen(c.diag_file, "w");
    if (!fp) { fprintf(stderr, "ERROR: cannot open %s\n", c.diag_file); return 1; }
    fprintf(fp, "t\tE_phi_kin\tE_theta_kin\tE_grad\tE_mass\tE_pot\tE_tgrad\tE_tmass\t"
                "E_coupling\tE_total\tphi_max\tP_max\tP_int\ttheta_rms");
    if (c.complex_phi)
        fprintf(fp, "\tQ_phi\tQ_theta\tQ_total\ts_max\tr_core\tomega_core\tQ_core\tthp1u\tthp1v\tthp2u\tthp2v");
    if (c.complex_gauge) fprintf(fp, "\tgauss_max\tgauss_l2\tE_em\tQ_flux");
    if (mf) fprintf(fp, "\tQ_C\tQ_Q\tQ_L\tQ_em");
    if (c.complex_phi) fprintf(fp, "\tQ_p0\tQ_p1\tQ_p2");
    fprintf(fp, "\n");

    const int n_steps = (int)lround(c.T / g->dt);
    int diag_every = (int)lround(c.diag_dt / g->dt); if (diag_every < 1) diag_every = 1;
    int snap_every = (int)lround(c.snap_dt / g->dt); if (snap_every < 1) snap_every = 1;
    scp_gpu_diag_out d;
    if ((rc = scp_gpu_diag(h, &d))) return fail("diag", rc);
    const double E0 = d.v[SCP_DIAG_E_TOTAL];
    printf("INIT: E_total=%.4e E_pot=%.4f phi_max=%.4f P_int=%.4e theta_rms=%.3e\n\n", E0, d.v[SCP_DIAG_E_POT],
           d.v[SCP_DIAG_PHI_MAX], d.v[SCP_DIAG_P_INT], d.v[SCP_DIAG_THETA_RMS]);
    diag_row(fp, 0.0, &d, c.complex_gauge, c.complex_phi, mf);

    int major = diag_every * 25;
    if (major > n_steps / 10) { major = (n_steps / 10 / diag_every) * diag_every; if (major < diag_every) major = diag_every; }
    const double wall0 = wall_now();
    int step = 0;
    while (step < n_steps) {
        /* advance to the next diag or snapshot step in one call */
        int next = n_steps;
        const int nd = (step / diag_every + 1) * diag_every, ns = (step / snap_every + 1) * snap_every;
        if (nd < next) next = nd;
        if (ns < next) next = ns;
        if ((rc = scp_gpu_step(h, next - step))) return fail("step", rc);
        if ((rc = snap_flush(&snap))) return fail("snapshot", rc);   /* its copy overlapped these steps */
        step = next;
        const double t = step * g->dt;
        if (step % snap_every == 0 && (rc = snap_start(&snap, t))) return fail("snapshot", rc);
        if (step % diag_every == 0) {
            if ((rc = scp_gpu_diag(h, &d))) return fail("diag", rc);
            diag_row(fp, t, &d, c.complex_gauge, c.complex_phi, mf);
            fflush(fp);
            if (step % major == 0) {
                const double wall = wall_now() - wall0;
                printf("t=%7.1f E=%.3e (drift %+.3f%%) Ep=%.1f phi=%.3f Q=%.6e ", t, d.v[SCP_DIAG_E_TOTAL],
                       100 * (d.v[SCP_DIAG_E_TOTAL] - E0) / (fabs(E0) + 1e-30), d.v[SCP_DIAG_E_POT],
                       d.v[SCP_DIAG_PHI_MAX], d.v[SCP_DIAG_Q_TOTAL]);
                if (c.complex_gauge) printf("gauss=%.1e E_em=%.3e ", d.v[SCP_DIAG_GAUSS_MAX], d.v[SCP_DIAG_E_EM]);
                printf("[%.0f%% %.1fs %.3fms/step]\n", 100.0 * step / n_steps, wall, 1000 * wall / step);
                fflush(stdout);
            }
        }
    }
    if ((rc = scp_gpu_sync(h))) return fail("sync", rc);
    const double wall = wall_now() - wall0;
    {   /* final frame unless the last step was (nearly) a snapshot step (scp_sim.c:3254-3259) */
        const int last = (n_steps / snap_every) * snap_every;
        if (n_steps - last > snap_every / 2 && (rc = snap_start(&snap, n_steps * g->dt))) return fail("snapshot", rc);
    }
    if ((rc = snap_close(&snap))) return fail("snapshot", rc);
    const uint32_t nf = sfa->total_frames;
    sfa_close(sfa);
    if ((rc = scp_gpu_diag(h, &d))) return fail("diag", rc);
    printf("\n=== COMPLETE ===\n");
    printf("E_total=%.4e (drift %.3f%%) E_pot=%.4f\n", d.v[SCP_DIAG_E_TOTAL],
           100 * (d.v[SCP_DIAG_E_TOTAL] - E0) / (fabs(E0) + 1e-30), d.v[SCP_DIAG_E_POT]);
    if (c.complex_phi)
        printf("Q_phi=%.6e Q_theta=%.6e Q_total=%.6e s_max=%.4e r_core=%.3f omega_core=%.4f Q_core=%.6e\n",
           d.v[SCP_DIAG_Q_PHI], d.v[SCP_DIAG_Q_THETA], d.v[SCP_DIAG_Q_TOTAL], d.v[SCP_DIAG_S_MAX],
           d.v[SCP_DIAG_R_CORE], d.v[SCP_DIAG_OMEGA_CORE], d.v[SCP_DIAG_Q_CORE]);
    if (c.complex_gauge)
        printf("gauss_max=%.3e gauss_l2=%.3e E_em=%.6e Q_flux=%.6e\n", d.v[SCP_DIAG_GAUSS_MAX],
               d.v[SCP_DIAG_GAUSS_L2], d.v[SCP_DIAG_E_EM], d.v[SCP_DIAG_Q_FLUX]);
    printf("SFA: %s (%u frames)\n", c.output, nf);
    printf("Wall: %.1fs (%.1f min) %.3fms/step\n", wall, wall / 60, n_steps ? 1000 * wall / n_steps : 0.0);
    fclose(fp);
    scp_gpu_free(h);
    free(g);
    return 0;
}
