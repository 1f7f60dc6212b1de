// serve.cuh -- continuous-batching request server (C ABI scp_srv_*).
//
// Included at the end of scp_gpu.cu: a request is an ordinary scp_gpu handle
// (its init does the upload, Gauss projection, precision conversion and the
// first half step), but once admitted its steps are taken by the server's
// multi-request launches instead of scp_gpu_step:
//
//   submit  -> queued (host copy of the columns; caller buffers may go)
//   load    -> a loader thread initialises queued requests (upload, Gauss
//              projection, precision conversion) while active slots and the
//              HBM budget allow, concurrently with the running chunks
//   poll    -> take the loaded requests in; rewrite the device request
//              tables; replay one chunk of
//              K steps as a CUDA graph (one persistent launch per step per
//              group of requests sharing precision, gauge mode and tile
//              shape; groups run on forked streams); retire finished
//              requests (diagnostics, optional snapshot, free)
//   result  -> final diagnostics (+ snapshot written at retirement)
//
// Requests that arrive while others run are admitted at the next chunk
// boundary, so the work of old and new requests overlaps on the device.
// The tile shape of each (grid size, gauge mode, precision) is chosen once by
// timing every compiled shape on a scratch state (autotune).
#pragma once

#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <deque>
#include <map>
#include <memory>
#include <tuple>
#include <vector>

namespace {

#ifndef SCP_SRV_OVERSUB
#define SCP_SRV_OVERSUB 8
#endif
constexpr int kSrvOversub = SCP_SRV_OVERSUB;
#ifndef SCP_SRV_SEG
#define SCP_SRV_SEG 16      // planes per work item in the multi-request launches
#endif

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct SrvReq {
    int64_t id = 0;
    scp_gpu_params p{};
    std::vector<double> cols;     // staged input, released at admission
    std::vector<const double *> borrowed;   // caller's columns (scp_srv_submit_borrowed)
    int64_t nsteps = 0;
    int state = 0;                // SCP_SRV_QUEUED / ACTIVE / DONE / FAILED
    int rc = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    long long s0 = 0, s1 = 0;
    scp_gpu *h = nullptr;
    int64_t bytes = 0;
    int group = -1;
    scp_gpu_diag_out diag{};
    void *const *out_cols = nullptr;
    int out_dtype = SCP_DTYPE_F64;
};

struct SrvGroup {
    int prec = 0, gauged = 0, shape = 1, pairs = 0, damp = 0;
    int grid = 0, threads = 0;
    size_t smem = 0;
    void *d_tab = nullptr;        // ReqTable<P> on the device
    void *h_tab = nullptr;        // pinned staging copy
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<SrvReq *> members;
};

template <class P>
size_t table_bytes() { return sizeof(ReqTable<P>); }

template <class P>
StepIO<P> req_io(scp_gpu *h, int par);

template <>
StepIO<F64> req_io<F64>(scp_gpu *h, int par) {
    const int in = h->cur ^ par;
    StepIO<F64> io;
    io.xin = h->X[in];
    io.xout = h->X[in ^ 1];
    io.loin = nullptr; io.loout = nullptr; io.tloin = nullptr; io.tloout = nullptr;
    io.win = h->W; io.wout = h->W; io.sout = h->S; io.flag = h->flag;
    return io;
}
template <>
StepIO<F32C> req_io<F32C>(scp_gpu *h, int par) {
    const int in = h->cur ^ par;
    StepIO<F32C> io;
    io.xin = h->X32[in];
    io.xout = h->X32[in ^ 1];
    io.loin = h->LO[in]; io.loout = h->LO[in ^ 1];
    io.tloin = h->TLO[in]; io.tloout = h->TLO[in ^ 1];
    io.win = h->W32; io.wout = h->W32; io.sout = h->S32; io.flag = h->flag;
    return io;
}

}  // namespace

struct scp_srv {
    scp_srv_config cfg{};
    cudaStream_t stream = nullptr;
    long long step = 0;
    int64_t next_id = 1;
    int64_t mem_in_use = 0;
    std::deque<SrvReq *> queue;
    std::vector<SrvReq *> active;
    std::map<int64_t, std::unique_ptr<SrvReq>> all;
    std::vector<std::unique_ptr<SrvGroup>> groups;
    std::map<std::tuple<int, int, int, int, int>, int> group_of;   // (prec, gauged, shape, pairs, damp) -> group
    std::map<std::tuple<int, int, int>, int> tuned;           // (N, gauged, prec) -> shape
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_groups = -1;                                    // group count the graph was built for
    int nsm = 0;
    int64_t chunks = 0;
    double t_admit = 0, t_autotune = 0, t_run = 0, t_retire = 0, t_wait = 0, t_launch = 0;
    double t_gpu = 0;                                         // device time of the chunks (events)
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool inflight = false;                                    // a chunk is running on the GPU
    // loader threads: queue -> (init) -> ready.  queue, ready, all, tuned,
    // the counters below and t_admit / t_autotune are guarded by mu.
    std::vector<std::thread> loaders;
    std::mutex mu;
    std::condition_variable cv;
    bool stop = false;
    std::deque<SrvReq *> ready;
    std::deque<SrvReq *> retiring;                            // finished, waiting for a retire thread
    std::vector<std::thread> retirers;
    int n_retiring = 0;                                       // queued or being retired
    int n_loading = 0;
    int n_held = 0;                                           // loading + ready + active
    int64_t mem_reserved = 0;                                 // footprint of the held requests
};

static int64_t srv_footprint(const scp_gpu_params &p) {
    const int64_t n3 = (int64_t)p.N * p.N * p.N;
    const int nf = p.complex_gauge ? 15 : 12;
    int64_t b = (p.precision_mode == SCP_PREC_FP64) ? 4LL * 8 * nf * n3
                                                   : 4LL * 4 * nf * n3 + 2LL * 24 * n3 + (p.complex_gauge ? 2LL * 12 * n3 : 0);
    return b + 8 * n3 + (int64_t)kRedMaxBlocks * 32 * 8;   // + snapshot staging + reduction partials
}

// time each compiled tile shape on a scratch state and keep the fastest
// (loader thread; the chunks of the active requests run meanwhile, so the
// shapes are compared under the same load)
static int srv_autotune(scp_srv *s, const scp_gpu_params &p, int *shape_out) {
    const auto key = std::make_tuple((int)p.N, (int)(p.complex_gauge != 0 && p.g_gauge != 0.0), (int)p.precision_mode);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tuned.find(key);
        if (it != s->tuned.end()) { *shape_out = it->second; return SCP_OK; }
    }
    if (!s->cfg.autotune) { *shape_out = 0; return SCP_OK; }
    const double t0 = now_s();
    const int64_t n3 = (int64_t)p.N * p.N * p.N;
    const int ncols = p.complex_gauge ? 30 : 24;
    std::vector<double> zero((size_t)n3, 0.0), bump((size_t)n3, 0.0);
    for (int64_t i = 0; i < n3; i++) bump[(size_t)i] = 1e-3 * (double)((i * 2654435761LL) % 1000) / 1000.0;
    std::vector<const double *> cols(ncols, zero.data());
    for (int c = 0; c < 6; c++) cols[c] = bump.data();   // phi and theta real parts: a non-trivial state
    double best = 1e300;
    int best_shape = 1;
    for (int shape = 1; shape < kNumShapes; shape++) {
        scp_gpu_params q = p;
        q.tile_variant = shape;
        q.gauss_project = 0;
        q.bc_type = 0;            // the scratch state need not be neutral
        q.damp_rate = 0.0;
        scp_gpu *h = nullptr;
        if (scp_gpu_init(&q, cols.data(), &h) != SCP_OK) continue;
        double ms = 0;
        scp_gpu_step(h, 3);
        const int rc = scp_gpu_time_steps(h, 10, &ms);
        scp_gpu_free(h);
        if (rc == SCP_OK && ms < best) { best = ms; best_shape = shape; }
    }
    *shape_out = best_shape;
    std::lock_guard<std::mutex> lk(s->mu);
    s->tuned[key] = best_shape;
    s->t_autotune += now_s() - t0;
    return SCP_OK;
}

static int srv_group(scp_srv *s, int prec, int gauged, int shape, int pairs, int damp, int *gidx) {
    const auto key = std::make_tuple(prec, gauged, shape, pairs, damp);
    auto it = s->group_of.find(key);
    if (it != s->group_of.end()) { *gidx = it->second; return SCP_OK; }
    auto g = std::make_unique<SrvGroup>();
    g->prec = prec; g->gauged = gauged; g->shape = shape; g->pairs = pairs; g->damp = damp;
    g->threads = kShapes[shape].tx * kShapes[shape].ty / (pairs ? 2 : 1);
    const void *fn;
    size_t tb;
    if (pairs) { fn = (const void *)multi2_fn(shape, gauged, damp, &g->smem); tb = table_bytes<F32C>(); }
    else if (prec == SCP_PREC_FP64) { fn = (const void *)multi_fn<F64>(shape, gauged, damp, &g->smem); tb = table_bytes<F64>(); }
    else { fn = (const void *)multi_fn<F32C>(shape, gauged, damp, &g->smem); tb = table_bytes<F32C>(); }
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g->smem));
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, g->threads, g->smem));
    if (occ < 1) return SCP_EUNSUPPORTED;
    // 8 CTAs per resident slot: CTAs retire every few work items, so the
    // start-up kernels of loading requests (higher stream priority) get SMs
    // between them instead of waiting for the end of a step
    g->grid = s->nsm * occ * kSrvOversub;
    CK(cudaMalloc(&g->d_tab, tb));
    CK(cudaMallocHost(&g->h_tab, tb));
    memset(g->h_tab, 0, tb);
    CK(cudaMemcpy(g->d_tab, g->h_tab, tb, cudaMemcpyHostToDevice));
    CK(cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming));
    s->groups.push_back(std::move(g));
    *gidx = (int)s->groups.size() - 1;
    s->group_of[key] = *gidx;
    return SCP_OK;
}

template <class P>
static void fill_table(scp_srv *s, SrvGroup *g) {
    ReqTable<P> *t = (ReqTable<P> *)g->h_tab;
    t->step = s->step;
    int items = 0, r = 0;
    for (SrvReq *q : g->members) {
        if (q->s1 <= s->step) continue;                  // finished, waiting to be retired
        ReqSlot<P> &slot = t->r[r++];
        slot.io[0] = req_io<P>(q->h, 0);
        slot.io[1] = req_io<P>(q->h, 1);
        slot.c = q->h->c;
        slot.tg = q->h->tg;
        slot.item0 = items;
        slot.s0 = q->s0;
        slot.s1 = q->s1;
        items += q->h->tg.nitems;
    }
    t->nreq = r;
    t->nitems = items;
}

// Segment length for the next chunk.  One launch advances every request by a
// step, so its duration is set by the slowest work item: cut every grid into
// segments of about the same number of planes (16) so items of large and
// small grids cost alike and the persistent CTAs stay balanced; split further
// only when the active set is too small to fill the GPU.
static void srv_plan(scp_srv *s) {
    long long items = 0;
    for (SrvReq *q : s->active)
        if (q->s1 > s->step) {
            const int N = q->h->N;
            items += (long long)q->h->tg.ntx * q->h->tg.nty * ((N + SCP_SRV_SEG - 1) / SCP_SRV_SEG);
        }
    const long long target = 6LL * s->nsm;
    int seg_planes = SCP_SRV_SEG;
    while (items < target && seg_planes > 4) { seg_planes /= 2; items *= 2; }
    for (SrvReq *q : s->active) {
        TileGrid &tg = q->h->tg;
        const int N = q->h->N;
        const int seg = N < seg_planes ? N : seg_planes;
        tg.seg = seg;
        tg.nseg = (N + seg - 1) / seg;
        tg.nitems = tg.ntx * tg.nty * tg.nseg;
    }
}

static int srv_upload_tables(scp_srv *s) {
    for (auto &g : s->groups) {
        size_t tb;
        if (g->prec == SCP_PREC_FP64) { fill_table<F64>(s, g.get()); tb = table_bytes<F64>(); }
        else { fill_table<F32C>(s, g.get()); tb = table_bytes<F32C>(); }
        CK(cudaMemcpyAsync(g->d_tab, g->h_tab, tb, cudaMemcpyHostToDevice, s->stream));
    }
    return SCP_OK;
}

static void srv_launch_group(const SrvGroup *g, int k) {
    size_t sm;
    if (g->pairs)
        multi2_fn(g->shape, g->gauged, g->damp, &sm)<<<g->grid, g->threads, g->smem, g->st>>>(
            (const ReqTable<F32C> *)g->d_tab, k);
    else if (g->prec == SCP_PREC_FP64)
        multi_fn<F64>(g->shape, g->gauged, g->damp, &sm)<<<g->grid, g->threads, g->smem, g->st>>>(
            (const ReqTable<F64> *)g->d_tab, k);
    else
        multi_fn<F32C>(g->shape, g->gauged, g->damp, &sm)<<<g->grid, g->threads, g->smem, g->st>>>(
            (const ReqTable<F32C> *)g->d_tab, k);
}

// one chunk: every group's K steps on its own stream, forked from and joined
// back to the server stream
static void srv_enqueue_chunk(scp_srv *s, cudaEvent_t fork) {
    cudaEventRecord(fork, s->stream);
    for (auto &g : s->groups) {
        cudaStreamWaitEvent(g->st, fork, 0);
        for (int k = 0; k < s->cfg.chunk_steps; k++) srv_launch_group(g.get(), k);
        cudaEventRecord(g->done, g->st);
        cudaStreamWaitEvent(s->stream, g->done, 0);
    }
}

// capture one chunk into a graph (rebuilt when the set of groups changes)
static int srv_build_graph(scp_srv *s) {
    if (s->exec) { cudaGraphExecDestroy(s->exec); s->exec = nullptr; }
    if (s->graph) { cudaGraphDestroy(s->graph); s->graph = nullptr; }
    cudaEvent_t fork;
    CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    srv_enqueue_chunk(s, fork);
    cudaError_t e = cudaStreamEndCapture(s->stream, &s->graph);
    cudaEventDestroy(fork);
    CK(e);
    CK(cudaGraphInstantiate(&s->exec, s->graph, 0));
    s->graph_groups = (int)s->groups.size();
    return SCP_OK;
}

// may the loader take the next queued request?  (caller holds mu)  A request
// larger than the whole budget still runs, alone.
static bool srv_can_load(const scp_srv *s) {
    if (s->queue.empty()) return false;
    if (s->n_held >= s->cfg.max_active || s->n_held >= kMaxReq) return false;
    const int64_t need = srv_footprint(s->queue.front()->p);
    return s->cfg.mem_budget_bytes <= 0 || s->n_held == 0 || s->mem_reserved + need <= s->cfg.mem_budget_bytes;
}

// Loader thread: initialise queued requests (tile autotune, upload, Gauss
// projection, conversion) on their own streams while the GPU runs chunks.
// Slots and budget are reserved when a request leaves the queue and given
// back at retirement.
static void srv_loader(scp_srv *s) {
    cudaSetDevice(s->cfg.device);
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess) t_stream_priority = greatest;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv.wait(lk, [s] { return s->stop || srv_can_load(s); });
        if (s->stop) return;
        SrvReq *q = s->queue.front();
        s->queue.pop_front();
        const int64_t need = srv_footprint(q->p);
        s->mem_reserved += need;
        s->n_held++;
        s->n_loading++;
        lk.unlock();
        const double t0 = now_s();
        int shape = 0;
        int rc = srv_autotune(s, q->p, &shape);
        q->p.tile_variant = shape;
        const int ncols = q->p.complex_gauge ? 30 : 24;
        const int64_t n3 = (int64_t)q->p.N * q->p.N * q->p.N;
        std::vector<const double *> cols(ncols);
        for (int c = 0; c < ncols; c++)
            cols[c] = q->borrowed.empty() ? q->cols.data() + (size_t)c * n3 : q->borrowed[c];
        q->t_admit = now_s();
        if (rc == SCP_OK) rc = scp_gpu_init(&q->p, cols.data(), &q->h);
        std::vector<double>().swap(q->cols);
        std::vector<const double *>().swap(q->borrowed);
        lk.lock();
        s->t_admit += now_s() - t0;
        s->n_loading--;
        q->bytes = need;
        if (rc != SCP_OK) {
            q->state = SCP_SRV_FAILED; q->rc = rc; q->t_done = now_s();
            s->mem_reserved -= need;
            s->n_held--;
        } else {
            s->ready.push_back(q);
        }
        s->cv.notify_all();
    }
}

// move loaded requests into the active set (poll thread), at most
// admit_per_poll of them per poll when that is set
static int srv_intake(scp_srv *s) {
    std::vector<SrvReq *> got;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const size_t cap = s->cfg.admit_per_poll > 0 ? (size_t)s->cfg.admit_per_poll : s->ready.size();
        while (!s->ready.empty() && got.size() < cap) {
            got.push_back(s->ready.front());
            s->ready.pop_front();
        }
    }
    int rc;
    for (size_t n = 0; n < got.size(); n++) {
        SrvReq *q = got[n];
        int gi;
        if ((rc = srv_group(s, q->p.precision_mode, q->h->gauged, q->h->shape, q->h->pairs,
                             damping_on(q->h) ? 1 : 0, &gi))) {
            std::lock_guard<std::mutex> lk(s->mu);    // hand the rest back; the caller sees the error
            for (size_t m = got.size(); m-- > n;) s->ready.push_front(got[m]);
            return rc;
        }
        q->group = gi;
        q->s0 = -1;                                           // set when its first chunk is launched
        q->s1 = -1;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            q->state = SCP_SRV_ACTIVE;
            s->mem_in_use += q->bytes;
        }
        s->groups[gi]->members.push_back(q);
        s->active.push_back(q);
    }
    return SCP_OK;
}

// Retire thread: a finished request's final (synchronous-momenta) step
// through the single-grid kernel, diagnostics, optional snapshot, free -- all
// on the request's own stream, while the poll thread keeps the chunks going.
static void srv_retirer(scp_srv *s) {
    cudaSetDevice(s->cfg.device);
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess) t_stream_priority = greatest;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv.wait(lk, [s] { return s->stop || !s->retiring.empty(); });
        if (s->retiring.empty()) return;                 // stop, nothing left
        SrvReq *q = s->retiring.front();
        s->retiring.pop_front();
        lk.unlock();
        const double t0 = now_s();
        scp_gpu *h = q->h;
        h->cur ^= (int)((q->nsteps - 1) & 1);
        h->steps = q->nsteps - 1;
        int rc = scp_gpu_step(h, 1);
        if (rc == SCP_OK) rc = scp_gpu_sync(h);
        const int rc2 = scp_gpu_diag(h, &q->diag);
        if (rc == SCP_OK) rc = rc2;
        if (q->out_cols && rc == SCP_OK) rc = scp_gpu_snapshot(h, q->out_dtype, q->out_cols);
        scp_gpu_free(h);
        q->h = nullptr;
        lk.lock();
        q->rc = rc;
        q->t_done = now_s();
        q->state = (rc == SCP_OK) ? SCP_SRV_DONE : SCP_SRV_FAILED;
        s->mem_in_use -= q->bytes;
        s->mem_reserved -= q->bytes;
        s->n_held--;
        s->n_retiring--;
        s->t_retire += now_s() - t0;
        s->cv.notify_all();
    }
}

// hand the requests whose table steps are done to the retire threads (they
// are no longer in the tables of the chunk in flight)
static int srv_retire(scp_srv *s) {
    std::vector<SrvReq *> keep, done;
    for (SrvReq *q : s->active) {
        if (q->s1 < 0 || q->s1 > s->step) keep.push_back(q);
        else done.push_back(q);
    }
    if (done.empty()) return SCP_OK;
    for (SrvReq *q : done) {
        auto &m = s->groups[q->group]->members;
        m.erase(std::remove(m.begin(), m.end(), q), m.end());
    }
    s->active.swap(keep);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (SrvReq *q : done) s->retiring.push_back(q);
        s->n_retiring += (int)done.size();
    }
    s->cv.notify_all();
    return SCP_OK;
}

extern "C" {

int scp_srv_create(const scp_srv_config *cfg, scp_srv **out) {
    if (!cfg || !out) return SCP_EINVAL;
    *out = nullptr;
    if (cfg->chunk_steps < 1 || cfg->chunk_steps > 4096 || cfg->max_active < 1) return SCP_EINVAL;
    if (cfg->loader_threads < 0 || cfg->loader_threads > 64) return SCP_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) return SCP_ENODEV;
    CK(cudaSetDevice(cfg->device));
    scp_srv *s = new scp_srv();
    s->cfg = *cfg;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, cfg->device);
    if (e != cudaSuccess) {
        delete s;
        snprintf(g_cuda_err, sizeof g_cuda_err, "%s", cudaGetErrorString(e));
        return SCP_ECUDA;
    }
    const int nload = cfg->loader_threads > 0 ? cfg->loader_threads : 4;
    for (int t = 0; t < nload; t++) s->loaders.emplace_back(srv_loader, s);
    for (int t = 0; t < 2; t++) s->retirers.emplace_back(srv_retirer, s);
    *out = s;
    return SCP_OK;
}

static int srv_submit(scp_srv *s, const scp_gpu_params *p, const double *const *host_cols, int64_t nsteps,
                      void *const *out_cols, int out_dtype, int64_t *id_out, bool borrow) {
    if (!s || !p || !host_cols || nsteps < 1 || !id_out) return SCP_EINVAL;
    int rc = validate(p);
    if (rc) return rc;
    if (p->device != s->cfg.device) return SCP_EINVAL;
    if (p->real_fields) return SCP_EUNSUPPORTED;   // the server takes complex and gauged requests
    if (p->complex_gauge && (p->higgs_v > 0 || p->g_gauge2 != 0)) return SCP_EUNSUPPORTED;   // fused kernels only
    if (p->n_fabrics == 3) return SCP_EUNSUPPORTED;
    auto q = std::make_unique<SrvReq>();
    q->p = *p;
    q->nsteps = nsteps;
    q->out_cols = out_cols;
    q->out_dtype = out_dtype;
    const int ncols = p->complex_gauge ? 30 : 24;
    const int64_t n3 = (int64_t)p->N * p->N * p->N;
    for (int c = 0; c < ncols; c++)
        if (!host_cols[c]) return SCP_EINVAL;
    if (borrow) {
        q->borrowed.assign(host_cols, host_cols + ncols);
    } else {
        q->cols.resize((size_t)ncols * n3);
        for (int c = 0; c < ncols; c++) memcpy(q->cols.data() + (size_t)c * n3, host_cols[c], sizeof(double) * n3);
    }
    q->state = SCP_SRV_QUEUED;
    q->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        q->id = s->next_id++;
        *id_out = q->id;
        s->queue.push_back(q.get());
        s->all[q->id] = std::move(q);
    }
    s->cv.notify_all();
    return SCP_OK;
}

int scp_srv_submit(scp_srv *s, const scp_gpu_params *p, const double *const *host_cols, int64_t nsteps,
                   void *const *out_cols, int out_dtype, int64_t *id_out) {
    return srv_submit(s, p, host_cols, nsteps, out_cols, out_dtype, id_out, false);
}

int scp_srv_submit_borrowed(scp_srv *s, const scp_gpu_params *p, const double *const *host_cols, int64_t nsteps,
                            void *const *out_cols, int out_dtype, int64_t *id_out) {
    return srv_submit(s, p, host_cols, nsteps, out_cols, out_dtype, id_out, true);
}

int scp_srv_poll(scp_srv *s, int *n_active, int *n_queued) {
    if (!s) return SCP_EINVAL;
    CK(cudaSetDevice(s->cfg.device));
    int rc;
    // 1. take in the requests the loader has finished; with nothing to run
    //    on the GPU, wait briefly for the first of them
    const double t0 = now_s();
    {
        std::unique_lock<std::mutex> lk(s->mu);
        if (!s->inflight && s->active.empty() && s->ready.empty() && (s->n_loading > 0 || srv_can_load(s)))
            s->cv.wait_for(lk, std::chrono::milliseconds(2), [s] { return !s->ready.empty(); });
    }
    if ((rc = srv_intake(s))) return rc;
    const double t1 = now_s();
    s->t_wait += t1 - t0;
    // 2. finish the chunk in flight
    if (s->inflight) {
        CK(cudaStreamSynchronize(s->stream));
        float ms = 0;
        if (cudaEventElapsedTime(&ms, s->ev0, s->ev1) == cudaSuccess) s->t_gpu += 1e-3 * ms;
        s->step += s->cfg.chunk_steps;
        s->chunks++;
        s->inflight = false;
    }
    const double t2 = now_s();
    s->t_run += t2 - t1;
    // 3. newly taken requests start with the next chunk
    bool work = false;
    for (SrvReq *q : s->active) {
        // the tables take all but the final step, which stores the synchronous
        // momenta and runs through the single-grid kernel at retirement
        if (q->s0 < 0) { q->s0 = s->step; q->s1 = s->step + q->nsteps - 1; }
        if (q->s1 > s->step) work = true;
    }
    // 4. launch the next chunk
    if (work) {
        srv_plan(s);
        if ((rc = srv_upload_tables(s))) return rc;
        if (s->cfg.use_graph && s->graph_groups != (int)s->groups.size() && (rc = srv_build_graph(s))) return rc;
        CK(cudaEventRecord(s->ev0, s->stream));
        if (s->cfg.use_graph) {
            CK(cudaGraphLaunch(s->exec, s->stream));
        } else {
            cudaEvent_t fork;
            CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
            srv_enqueue_chunk(s, fork);
            cudaEventDestroy(fork);
            CK(cudaGetLastError());
        }
        CK(cudaEventRecord(s->ev1, s->stream));
        s->inflight = true;
    }
    s->t_launch += now_s() - t2;
    // 5. retire the requests that finished in the chunk just completed, while
    //    the next one runs (they are no longer in the tables)
    if ((rc = srv_retire(s))) return rc;
    if (!s->inflight && s->active.empty() && s->stream) CK(cudaStreamSynchronize(s->stream));
    int queued, retiring;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        // nothing else to do: let the retire threads finish before reporting
        if (!s->inflight && s->active.empty() && s->n_retiring > 0)
            s->cv.wait_for(lk, std::chrono::milliseconds(2), [s] { return s->n_retiring == 0; });
        queued = (int)(s->queue.size() + s->ready.size()) + s->n_loading;
        retiring = s->n_retiring;
    }
    if (n_active) *n_active = (int)s->active.size() + retiring;   // retiring requests still count as active
    if (n_queued) *n_queued = queued;
    return SCP_OK;
}

int scp_srv_status(scp_srv *s, int64_t id, scp_srv_request_info *info) {
    if (!s || !info) return SCP_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return SCP_EINVAL;
    const SrvReq *q = it->second.get();
    memset(info, 0, sizeof *info);
    info->state = q->state;
    info->rc = q->rc;
    info->t_submit = q->t_submit;
    info->t_admit = q->t_admit;
    info->t_done = q->t_done;
    info->nsteps = q->nsteps;
    info->N = q->p.N;
    info->tile_variant = q->p.tile_variant;
    return SCP_OK;
}

int scp_srv_result(scp_srv *s, int64_t id, scp_gpu_diag_out *diag) {
    if (!s || !diag) return SCP_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return SCP_EINVAL;
    const SrvReq *q = it->second.get();
    if (q->state == SCP_SRV_QUEUED || q->state == SCP_SRV_ACTIVE) return SCP_EBUSY;
    *diag = q->diag;
    return q->rc;
}

int scp_srv_stats(scp_srv *s, scp_srv_stats_t *st) {
    if (!s || !st) return SCP_EINVAL;
    memset(st, 0, sizeof *st);
    st->step = s->step;
    st->chunks = s->chunks;
    st->n_active = (int)s->active.size();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        st->mem_in_use = s->mem_in_use;
        st->n_active += s->n_retiring;
        st->t_retire = s->t_retire;
        st->n_queued = (int)(s->queue.size() + s->ready.size()) + s->n_loading;
        st->t_admit = s->t_admit - s->t_autotune;   // loader thread, overlapped with the chunks
        st->t_autotune = s->t_autotune;
    }
    st->n_groups = (int)s->groups.size();
    st->t_run = s->t_run;
    st->t_wait = s->t_wait;
    st->t_launch = s->t_launch;
    st->t_gpu = s->t_gpu;
    return SCP_OK;
}

void scp_srv_free(scp_srv *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (auto &t : s->loaders)
        if (t.joinable()) t.join();
    for (auto &t : s->retirers)   // they drain the retire queue before leaving
        if (t.joinable()) t.join();
    cudaSetDevice(s->cfg.device);
    for (SrvReq *q : s->ready)
        if (q->h) scp_gpu_free(q->h);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (SrvReq *q : s->active)
        if (q->h) scp_gpu_free(q->h);
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    for (auto &g : s->groups) {
        cudaFree(g->d_tab);
        cudaFreeHost(g->h_tab);
        if (g->st) cudaStreamDestroy(g->st);
        if (g->done) cudaEventDestroy(g->done);
    }
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

}  // extern "C"
