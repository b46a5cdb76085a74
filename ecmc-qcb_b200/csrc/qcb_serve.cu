// qcb_serve.cu -- continuous-batching Wilson-flow measurement server.
//
// Requests (a configuration of any L^4 size, a flow step, a number of measured steps) arrive
// through qcb_serve_submit from any host thread.  A scheduler thread owns the GPU work:
//   * admission: requests leave the FIFO in order as soon as the HBM budget (and the active
//     limit) leaves room for their flowed field, RK3 buffers and measurements; memory comes from
//     the server's own stream-ordered pool and returns to it when a request completes;
//   * one scheduler tick measures Q/E of every resident request and then advances every
//     resident request by n_rk RK3 steps.  Requests below kBigVh half-sites share one batched
//     clover launch (with a per-request finalize) and three persistent launches per RK3 step over
//     the tile work list of all of them, so requests that arrive while others are on the GPU
//     share the same launches; a request of kBigVh half-sites or more fills the GPU by itself and
//     runs the single-lattice kernels (geometry in kernel parameters, no per-tile descriptor
//     lookups).  Big requests run on one stream and the shared launches of the small ones on a
//     second, so the small requests' short launches overlap the big requests' kernels;
//   * a request that has taken its last measurement is copied back, frees its memory and is
//     handed to qcb_serve_poll with its submit and completion times.
// Per-request results do not depend on the other requests in the mix: every link and every
// per-request reduction is computed exactly as it would be alone.
// Replaces the measurement loop of topo_charge_flowed (src/observables/observables_mpi.cpp:159-186)
// driven once per configuration by the reference's drivers (src/bin/gauge_hb_cb.cpp:184-197).
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "qcb_internal.h"
#include "qcb_ops.h"

// Requests take every measurement from a measuring stage 1 (clover halves), as qcb_flow_measure
// does: that of the RK3 step that follows it, or for the last one a stage 1 whose output is left
// unused; 0 measures with clover passes.
#ifndef QCB_SERVE_FUSED_MEAS
#define QCB_SERVE_FUSED_MEAS 1
#endif

using namespace qcb;

namespace {

struct Request {
    uint64_t id = 0;
    Geom g{};
    double eps = 0.02;
    int n_steps = 1;
    std::vector<double> input;  // host AoS FP64 links, dropped after upload
    std::vector<double> tqe;    // 3 * n_steps results
    double t_submit = 0, t_admit = 0, t_done = 0;
    void* buf = nullptr;  // W, W', Z, measurements in one allocation
    size_t bytes = 0;
    size_t off_out = 0, off_z = 0, off_meas = 0;
    size_t off_halves = 0;  // small requests: clover halves of the tiled measuring stage 1 (0: none)
    int tick0 = 0;
    int flip = 0;
    cudaStream_t st = nullptr;  // the stream of all its work (big or small requests' stream)
    double* meas_slot = nullptr;  // a big request's slot of this tick, filled by its next stage 1
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Requests with at least this many half-sites (L >= 24 for L^4) run their own single-lattice
// launches; the choice depends on the request alone, so its result does not depend on the mix.
constexpr int64_t kBigVh = (int64_t)1 << 17;
bool is_big(const Request* r) { return r->g.Vh >= kBigVh; }

}  // namespace

struct qcb_server_s {
    size_t budget = 0;
    int prec = 32, store = 0, fmt = 2, max_active = 1 << 30, n_rk = 1;
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> pending, done;
    std::vector<Request*> active;
    std::vector<Request*> small, big;  // the active set split by size (rebuild)
    double* big_partials = nullptr;
    size_t big_partials_cap = 0;
    char* halves = nullptr;  // clover halves of a big request's measuring stage 1 (shared: one stream)
    size_t halves_cap = 0;
    size_t bytes_in_use = 0, bytes_peak = 0;
    uint64_t submitted = 0, completed = 0;
    bool stop = false;
    int err = QCB_OK;
    std::string errmsg;
    std::thread th;
    cudaStream_t stream = nullptr;        // big requests (single-lattice kernels)
    cudaStream_t stream_small = nullptr;  // small requests (shared tiled launches)
    cudaEvent_t ev_layout = nullptr;      // last conversion out of the shared upload staging
    bool layout_pending = false;
    cudaMemPool_t pool = nullptr;
    // work list of the active set
    std::vector<LatDesc> desc;
    LatDesc* d_desc = nullptr;
    size_t desc_cap = 0;
    int* d_tile_lat = nullptr;
    size_t tile_cap = 0;
    int nb_total = 0;
    double* partials = nullptr;
    size_t partials_cap = 0;
    double2* staging = nullptr;
    size_t staging_cap = 0;
    // CUDA graphs of the small requests' shared launches: one tick's measurement (clover pass,
    // per-request finalize, tick counter) and its n_rk RK3 steps, captured for the resident set of
    // `version` and the buffer parity the tick starts from, replayed while the set is unchanged
    std::atomic<bool> graphs{true};
    uint64_t version = 0;       // bumped by every rebuild of the work list
    uint64_t version_ticks = 0;  // ticks measured with the current version
    struct TickGraph {
        cudaGraphExec_t exec = nullptr;
        uint64_t version = 0;
        int kernels = 0;
    } gmeas[2], gflow[2];
    int* d_tick = nullptr;  // the tick the device's finalize kernels write (advanced on the device)
    int tick_dev = 0;       // the value d_tick holds once the enqueued work has run
    int tick_copy = 0;      // host source of a d_tick reset
    // counters of the two request sets, which tick at their own pace: measurements taken (slot
    // index base) and RK3 steps executed (buffer parity) of the small set, then of the big set
    int tick = 0;
    uint64_t nflow = 0;
    int tick_b = 0;
    uint64_t nflow_b = 0;
    uint64_t ticks = 0;
    int active_peak = 0;
    double busy = 0.0;
    std::chrono::steady_clock::time_point t0;
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

// Per-request deterministic sums of (q, e) partials, m tiles a lattice block of sites, stored in the
// request's slot of this tick: meas[(tick - tick0) * 3 + k] = (Q, sum e) (k = 0, 1; slot k = 2 is
// the plaquette sum, which only the single-lattice path measures).
__global__ void k_meas_finalize(const LatDesc* __restrict__ lats, const double* __restrict__ partials,
                                const int* __restrict__ d_tick, int m) {
    __shared__ double sm[256];
    const int tick = *d_tick;
    const LatDesc* d = lats + blockIdx.x;
    const int t0 = m * d->nb_begin, nt = m * d->nb;
    for (int k = 0; k < 2; k++) {
        double acc = 0.0;
        for (int i = threadIdx.x; i < nt; i += 256) acc += partials[(size_t)(t0 + i) * 2 + k];
        sm[threadIdx.x] = acc;
        __syncthreads();
        for (int s = 128; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) d->meas[(size_t)(tick - d->tick0) * 3 + k] = sm[0];
        __syncthreads();
    }
}

// Advances the device tick counter after a tick's finalize kernels have read it.
__global__ void k_tick_bump(int* d_tick) { *d_tick += 1; }

int set_error(qcb_server_s* s, int code, const std::string& msg) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->err == QCB_OK) {
        s->err = code;
        s->errmsg = msg;
    }
    s->cv_done.notify_all();
    return code;
}

bool cuda_ok(qcb_server_s* s, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(s, e == cudaErrorMemoryAllocation ? QCB_ENOMEM : QCB_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

template <typename T>
bool grow(qcb_server_s* s, T** p, size_t* cap, size_t n) {
    if (*cap >= n) return true;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    size_t m = std::max<size_t>(n, 1024);
    if (!cuda_ok(s, cudaMalloc((void**)p, m * sizeof(T)), "server work-list buffer")) return false;
    *cap = m;
    return true;
}

// Rebuilds the descriptors and tile map of the active set.
bool rebuild(qcb_server_s* s) {
    s->version++;
    s->version_ticks = 0;
    s->desc.clear();
    s->small.clear();
    s->big.clear();
    for (Request* r : s->active) (is_big(r) ? s->big : s->small).push_back(r);
    std::vector<int> tile_lat;
    int nb = 0;
    for (size_t i = 0; i < s->small.size(); i++) {
        Request* r = s->small[i];
        LatDesc d;
        memset(&d, 0, sizeof(d));
        d.g = r->g;
        d.links = r->buf;
        d.links_out = (char*)r->buf + r->off_out;
        d.z = (char*)r->buf + r->off_z;
        d.meas = (double*)((char*)r->buf + r->off_meas);
        d.halves = r->off_halves ? (char*)r->buf + r->off_halves : nullptr;
        d.eps = r->eps;
        d.nb_begin = nb;
        d.nb = (int)((r->g.Vh + TILE - 1) / TILE);
        d.flip = r->flip;
        d.tick0 = r->tick0;
        for (int k = 0; k < d.nb; k++) tile_lat.push_back((int)i);
        nb += d.nb;
        s->desc.push_back(d);
    }
    s->nb_total = nb;
    if (s->desc.empty()) return true;
    if (!grow(s, &s->d_desc, &s->desc_cap, s->desc.size())) return false;
    if (!grow(s, &s->d_tile_lat, &s->tile_cap, tile_lat.size())) return false;
    if (!grow(s, &s->partials, &s->partials_cap, (size_t)12 * nb)) return false;
    // pageable sources: the copies are staged before the calls return
    if (!cuda_ok(s, cudaMemcpyAsync(s->d_desc, s->desc.data(), sizeof(LatDesc) * s->desc.size(),
                                    cudaMemcpyHostToDevice, s->stream_small), "descriptor upload"))
        return false;
    return cuda_ok(s, cudaMemcpyAsync(s->d_tile_lat, tile_lat.data(), sizeof(int) * tile_lat.size(),
                                      cudaMemcpyHostToDevice, s->stream_small), "tile map upload");
}

// Admission on the request's stream; the upload into the shared staging waits until the previous
// admission's conversion (on either stream) has read it.
bool admit(qcb_server_s* s, Request* r) {
    r->t_admit = s->now();
    r->st = is_big(r) ? s->stream : s->stream_small;
    if (!cuda_ok(s, cudaMallocFromPoolAsync(&r->buf, r->bytes, s->pool, r->st), "request allocation")) return false;
    const size_t nd = (size_t)r->g.V * 72;
    if (!grow(s, &s->staging, &s->staging_cap, nd / 2)) return false;
    if (s->layout_pending && !cuda_ok(s, cudaStreamWaitEvent(r->st, s->ev_layout, 0), "upload order")) return false;
    if (!cuda_ok(s, cudaMemcpyAsync(s->staging, r->input.data(), nd * sizeof(double), cudaMemcpyHostToDevice, r->st),
                 "request upload"))
        return false;
    if (!cuda_ok(s, fmt_ops(s->fmt).aos_to_soa(r->g, s->staging, r->buf, 0, r->st), "request layout")) return false;
    note_launches(1);
    if (!cuda_ok(s, cudaEventRecord(s->ev_layout, r->st), "layout event")) return false;
    s->layout_pending = true;
    std::vector<double>().swap(r->input);
    r->tick0 = is_big(r) ? s->tick_b : s->tick;
    r->flip = (int)((is_big(r) ? s->nflow_b : s->nflow) & 1);  // current links in buffer A
    return true;
}

bool finish(qcb_server_s* s, Request* r) {
    std::vector<double> meas((size_t)r->n_steps * 3);
    if (!cuda_ok(s, cudaMemcpyAsync(meas.data(), (char*)r->buf + r->off_meas, meas.size() * sizeof(double),
                                    cudaMemcpyDeviceToHost, r->st), "result readback"))
        return false;
    if (!cuda_ok(s, cudaFreeAsync(r->buf, r->st), "request free")) return false;
    if (!cuda_ok(s, cudaStreamSynchronize(r->st), "result sync")) return false;
    r->buf = nullptr;
    r->tqe.resize((size_t)r->n_steps * 3);
    double t = 0.0;
    for (int k = 0; k < r->n_steps; k++) {
        r->tqe[3 * k] = t;
        r->tqe[3 * k + 1] = meas[3 * k];
        r->tqe[3 * k + 2] = meas[3 * k + 1] / (double)r->g.V;
        for (int j = 0; j < s->n_rk; j++) t += r->eps;
    }
    r->t_done = s->now();
    return true;
}

// Current links of a request: buffer A when an even number of RK3 steps has run since its
// admission, else buffer B (the rule the tiled kernels apply through flip ^ flip_xor).
void* current_links(const Request* r, int flip_xor) {
    return ((r->flip ^ flip_xor) & 1) ? (char*)r->buf + r->off_out : r->buf;
}

// Clover Q/E (and plaquette) of a big request with the single-lattice kernel, summed into its
// measurement slot of this tick.
bool measure_big(qcb_server_s* s, Request* r, int flip_xor) {
    const unsigned nbx = clover_blocks(r->g.Vh);
    if (!grow(s, &s->big_partials, &s->big_partials_cap, (size_t)nbx * 6 * 3)) return false;
    if (!cuda_ok(s, fmt_ops(s->fmt).clover(r->g, current_links(r, flip_xor), s->big_partials, nbx, s->stream),
                 "clover launch"))
        return false;
    double* slot = (double*)((char*)r->buf + r->off_meas) + (size_t)(s->tick_b - r->tick0) * 3;
    k_finalize<<<1, 256, 0, s->stream>>>(s->big_partials, (int)(nbx * 6), 3, 0u, slot);
    note_launches(2);
    return cuda_ok(s, cudaGetLastError(), "measure finalize");
}

// Stage 1 of a big request's RK3 step that also measures its input, into r->meas_slot: the
// measuring stage 1, the per-site sum of the clover halves and the finalize of qcb_flow_measure
// (same kernels, same partial counts), so a big request's rows equal the plain measured flow's.
bool flow_big_meas(qcb_server_s* s, Request* r, int flip_xor, int rep) {
    const int f = (r->flip ^ flip_xor) & 1;
    void* a = r->buf;
    void* b = (char*)r->buf + r->off_out;
    const unsigned nb = halves_blocks(r->g.Vh);
    if (!grow(s, &s->halves, &s->halves_cap, halves_bytes(s->fmt, r->g.Vh))) return false;
    if (!grow(s, &s->big_partials, &s->big_partials_cap, (size_t)nb * 3)) return false;
    const FmtOps& o = fmt_ops(s->fmt);
    if (!cuda_ok(s, o.flow1_meas(r->g, (f & 1) ? b : a, (f & 1) ? a : b, (char*)r->buf + r->off_z, r->eps, rep,
                                 s->halves, s->stream),
                 "flow launch"))
        return false;
    if (!cuda_ok(s, o.clover_halves(r->g, s->halves, s->big_partials, nb, s->stream), "clover launch")) return false;
    k_finalize<<<1, 256, 0, s->stream>>>(s->big_partials, (int)nb, 3, 0u, r->meas_slot);
    note_launches(3);
    r->meas_slot = nullptr;
    return cuda_ok(s, cudaGetLastError(), "measure finalize");
}

// One RK3 stage of a big request: stage s reads buffer A when (f + s - 1) is even (f = number
// of RK3 steps since admission, mod 2) and writes the other buffer.
bool flow_big(qcb_server_s* s, Request* r, int stage, int flip_xor, int rep) {
    const int f = (r->flip ^ flip_xor) & 1;
    void* a = r->buf;
    void* b = (char*)r->buf + r->off_out;
    const bool in_b = ((f + stage - 1) & 1) != 0;
    note_launches(1);
    return cuda_ok(s, fmt_ops(s->fmt).flow1(r->g, in_b ? b : a, in_b ? a : b, (char*)r->buf + r->off_z, r->eps, stage,
                                            rep, s->stream),
                   "flow launch");
}

// The small requests' measurement of one tick, into each request's slot of the device tick, and the
// tick counter advanced.  It is the measuring stage 1 of the tick's first RK3 step (clover halves;
// a request taking its last measurement runs it too, and its flow output is left unused) and the
// halves' per-tile sums, as qcb_flow_measure measures; without QCB_SERVE_FUSED_MEAS, a batched
// clover pass.  Returns the kernels launched (or -1).
int small_measure(qcb_server_s* s, const WorkList& w, int fx, int rep) {
    const FmtOps& o = fmt_ops(s->fmt);
    int m = 6;
    if (QCB_SERVE_FUSED_MEAS) {
        if (!cuda_ok(s, o.flow_tiles1_meas(w, fx, rep, s->stream_small), "flow launch")) return -1;
        if (!cuda_ok(s, o.halves_tiles(w, s->partials, s->stream_small), "clover launch")) return -1;
        m = 2;
    } else if (!cuda_ok(s, o.clover_tiles(w, fx, s->partials, s->stream_small), "clover launch")) {
        return -1;
    }
    k_meas_finalize<<<(unsigned)s->small.size(), 256, 0, s->stream_small>>>(s->d_desc, s->partials, s->d_tick, m);
    k_tick_bump<<<1, 1, 0, s->stream_small>>>(s->d_tick);
    return cuda_ok(s, cudaGetLastError(), "measure finalize") ? (QCB_SERVE_FUSED_MEAS ? 4 : 3) : -1;
}
// The small requests' n_rk RK3 steps, from buffer parity f0 (stage 1 of the first one ran in the
// measurement).
int small_flow(qcb_server_s* s, const WorkList& w, int f0, int rep) {
    for (int k = 0; k < s->n_rk; k++)
        for (int stage = (QCB_SERVE_FUSED_MEAS && k == 0) ? 2 : 1; stage <= 3; stage++)
            if (!cuda_ok(s, fmt_ops(s->fmt).flow(w, stage, (f0 + k) & 1, rep, s->stream_small), "flow launch"))
                return -1;
    return 3 * s->n_rk - (QCB_SERVE_FUSED_MEAS ? 1 : 0);
}

// Runs body (small_measure or small_flow) for parity fx: plainly on the first tick of a resident
// set (or with graphs off), else by replaying the graph captured from the same set and parity.
template <class Body>
bool small_run(qcb_server_s* s, qcb_server_s::TickGraph cache[2], int fx, Body body) {
    if (!s->graphs.load() || s->version_ticks < 1) {
        const int k = body();
        if (k < 0) return false;
        note_launches(k);
        return true;
    }
    qcb_server_s::TickGraph& g = cache[fx];
    if (!g.exec || g.version != s->version) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = qcb_server_s::TickGraph{};
        cudaGraph_t graph = nullptr;
        if (!cuda_ok(s, cudaStreamBeginCapture(s->stream_small, cudaStreamCaptureModeThreadLocal), "tick capture"))
            return false;
        const int k = body();
        const cudaError_t e = cudaStreamEndCapture(s->stream_small, &graph);
        if (k < 0) {
            if (graph) cudaGraphDestroy(graph);
            return false;
        }
        if (!cuda_ok(s, e, "tick capture end")) return false;
        const cudaError_t ei = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (!cuda_ok(s, ei, "tick graph instantiate")) {
            g.exec = nullptr;
            return false;
        }
        g.version = s->version;
        g.kernels = k;
    }
    if (!cuda_ok(s, cudaGraphLaunch(g.exec, s->stream_small), "tick graph launch")) return false;
    note_launches(g.kernels);
    return true;
}

void drop_tick_graphs(qcb_server_s* s) {
    for (auto* c : {s->gmeas, s->gflow})
        for (int i = 0; i < 2; i++) {
            if (c[i].exec) cudaGraphExecDestroy(c[i].exec);
            c[i] = qcb_server_s::TickGraph{};
        }
}

// Small-request ticks a scheduler round runs beside one big-request tick, so that the two streams
// get similar work and a small request does not wait for the big ones' steps: the big set's sites
// over the small set's (the shared tile kernels cost about a third more a site), 1 to 8.
constexpr int kMaxSmallTicks = 8;
int small_ticks(const qcb_server_s* s) {
    if (s->big.empty() || s->small.empty()) return 1;
    double vb = 0.0, vs = 0.0;
    for (const Request* r : s->big) vb += (double)r->g.V;
    for (const Request* r : s->small) vs += (double)r->g.V;
    return std::min(kMaxSmallTicks, std::max(1, (int)(vb / (1.3 * vs) + 0.5)));
}

WorkList small_worklist(const qcb_server_s* s) {
    WorkList w;
    w.lats = s->d_desc;
    w.tile_lat = s->d_tile_lat;
    w.nb_total = s->nb_total;
    w.nlat = (int)s->small.size();
    return w;
}

// Requests that took their last measurement leave: results read back, memory returned, published.
bool retire(qcb_server_s* s, const std::vector<Request*>& leaving) {
    if (leaving.empty()) return true;
    for (Request* r : leaving)
        if (!finish(s, r)) return false;
    std::vector<Request*> staying;
    for (Request* r : s->active)
        if (std::find(leaving.begin(), leaving.end(), r) == leaving.end()) staying.push_back(r);
    s->active.swap(staying);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (Request* r : leaving) {
            s->bytes_in_use -= r->bytes;
            s->done.push_back(r);
            s->completed++;
        }
        s->cv_done.notify_all();
    }
    return rebuild(s);
}

// One tick of the big requests (single-lattice kernels on the big stream): measure each at its
// current step, retire those done, advance the others by n_rk RK3 steps.
bool big_tick(qcb_server_s* s, int rep) {
    const int fx = (int)(s->nflow_b & 1);
    bool ok = true;
    // a big request that flows on after this measurement takes it from its next stage 1; its last
    // measurement runs a measuring stage 1 now, whose output is left unused
    for (Request* r : s->big) {
        if (QCB_SERVE_FUSED_MEAS) {
            r->meas_slot = (double*)((char*)r->buf + r->off_meas) + (size_t)(s->tick_b - r->tick0) * 3;
            if (s->tick_b - r->tick0 == r->n_steps - 1) ok = ok && flow_big_meas(s, r, fx, rep);
        } else {
            ok = ok && measure_big(s, r, fx);
        }
    }
    if (!ok) return false;
    std::vector<Request*> leaving;
    for (Request* r : s->big)
        if (s->tick_b - r->tick0 == r->n_steps - 1) leaving.push_back(r);
    s->tick_b++;
    if (!retire(s, leaving)) return false;
    const int f0 = (int)(s->nflow_b & 1);
    for (int k = 0; k < s->n_rk && ok; k++) {
        const int f = (f0 + k) & 1;
        for (int stage = 1; stage <= 3 && ok; stage++)
            for (Request* r : s->big)
                ok = ok && (stage == 1 && r->meas_slot ? flow_big_meas(s, r, f, rep) : flow_big(s, r, stage, f, rep));
    }
    s->nflow_b += (uint64_t)s->n_rk;
    return ok;
}

// One tick of the small requests (shared tile launches on the small stream, replayed from graphs
// while the set is unchanged): measure, retire those done, advance the others.
bool small_tick(qcb_server_s* s, int rep) {
    WorkList w = small_worklist(s);
    const int fx = (int)(s->nflow & 1);
    if (s->tick_dev != s->tick) {  // a reset of the set left the device counter behind
        s->tick_copy = s->tick;
        if (!cuda_ok(s, cudaMemcpyAsync(s->d_tick, &s->tick_copy, sizeof(int), cudaMemcpyHostToDevice,
                                        s->stream_small), "tick counter"))
            return false;
    }
    if (!small_run(s, s->gmeas, fx, [&] { return small_measure(s, w, fx, rep); })) return false;
    s->tick_dev = s->tick + 1;
    s->version_ticks++;
    std::vector<Request*> leaving;
    for (Request* r : s->small)
        if (s->tick - r->tick0 == r->n_steps - 1) leaving.push_back(r);
    s->tick++;
    if (!retire(s, leaving)) return false;
    if (!s->small.empty()) {
        w = small_worklist(s);
        const int f0 = (int)(s->nflow & 1);
        if (!small_run(s, s->gflow, f0, [&] { return small_flow(s, w, f0, rep); })) return false;
    }
    s->nflow += (uint64_t)s->n_rk;
    return true;
}

void scheduler(qcb_server_s* s) {
    cudaSetDevice(s->device);
    const int rep = needs_reproject(s->prec, s->store);
    while (true) {
        std::vector<Request*> fresh;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty() || !s->active.empty(); });
            if (s->stop || s->err != QCB_OK) break;
            while (!s->pending.empty() && (int)s->active.size() < s->max_active &&
                   s->bytes_in_use + s->pending.front()->bytes <= s->budget) {
                Request* r = s->pending.front();
                s->pending.pop_front();
                s->bytes_in_use += r->bytes;
                s->bytes_peak = std::max(s->bytes_peak, s->bytes_in_use);
                fresh.push_back(r);
            }
        }
        const double tb = s->now();
        bool ok = true;
        for (Request* r : fresh) {
            ok = ok && admit(s, r);
            s->active.push_back(r);
        }
        if (ok && !fresh.empty()) ok = rebuild(s);
        if (!ok) break;
        if (s->active.empty()) continue;
        const int n_active = (int)s->active.size();
        // one round: a tick of the big requests and m ticks of the small ones
        const int m = small_ticks(s);
        if (!s->big.empty()) ok = big_tick(s, rep);
        for (int j = 0; ok && j < m && !s->small.empty(); j++) ok = small_tick(s, rep);
        if (!ok) break;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->ticks++;
            s->active_peak = std::max(s->active_peak, n_active);
            s->busy += s->now() - tb;
        }
    }
    cudaStreamSynchronize(s->stream);
    cudaStreamSynchronize(s->stream_small);
    drop_tick_graphs(s);
}

}  // namespace

extern "C" {

int qcb_serve_create(size_t hbm_budget_bytes, int prec, int store, int n_rk, int max_active, qcb_server* out) {
    if (!out || hbm_budget_bytes == 0 || n_rk < 1) return fail(QCB_EINVAL, "serve: invalid argument");
    if (prec != QCB_PREC_F64 && prec != QCB_PREC_F32) return fail(QCB_EINVAL, "prec must be 64 or 32");
    if (store != QCB_STORE_18 && store != QCB_STORE_12) return fail(QCB_EINVAL, "store must be 0 or 1");
    qcb_server_s* s = new (std::nothrow) qcb_server_s();
    if (!s) return fail(QCB_ENOMEM, "host allocation");
    s->budget = hbm_budget_bytes;
    s->prec = prec;
    s->store = store;
    s->fmt = fmt_of(prec, store);
    s->n_rk = n_rk;
    s->max_active = max_active > 0 ? max_active : (1 << 30);
    s->t0 = std::chrono::steady_clock::now();
    cudaGetDevice(&s->device);
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream_small, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_layout, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_tick, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(s->d_tick, 0, sizeof(int));
    if (e == cudaSuccess) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = s->device;
        e = cudaMemPoolCreate(&s->pool, &props);
    }
    if (e == cudaSuccess) {
        uint64_t keep = hbm_budget_bytes;
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e != cudaSuccess) {
        int r = fail(QCB_ECUDA, "serve create: %s", cudaGetErrorString(e));
        qcb_serve_destroy(s);
        return r;
    }
    s->th = std::thread(scheduler, s);
    *out = s;
    return QCB_OK;
}

int qcb_serve_destroy(qcb_server s) {
    if (!s) return QCB_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->th.joinable()) s->th.join();
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->stream_small) cudaStreamSynchronize(s->stream_small);
    for (Request* r : s->active) {
        if (r->buf) cudaFreeAsync(r->buf, r->st ? r->st : s->stream);
        delete r;
    }
    for (Request* r : s->pending) delete r;
    for (Request* r : s->done) delete r;
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->stream_small) cudaStreamSynchronize(s->stream_small);
    if (s->ev_layout) cudaEventDestroy(s->ev_layout);
    if (s->d_tick) cudaFree(s->d_tick);
    if (s->d_desc) cudaFree(s->d_desc);
    if (s->d_tile_lat) cudaFree(s->d_tile_lat);
    if (s->partials) cudaFree(s->partials);
    if (s->big_partials) cudaFree(s->big_partials);
    if (s->halves) cudaFree(s->halves);
    if (s->staging) cudaFree(s->staging);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->stream_small) cudaStreamDestroy(s->stream_small);
    delete s;
    return QCB_OK;
}

int qcb_serve_set_option(qcb_server s, int option, int value) {
    if (!s) return fail(QCB_EINVAL, "null server");
    if (option == QCB_SERVE_GRAPHS) {
        s->graphs.store(value != 0);
        return QCB_OK;
    }
    return fail(QCB_EINVAL, "unknown server option %d", option);
}

double qcb_serve_now(qcb_server s) { return s ? s->now() : 0.0; }

int qcb_serve_submit(qcb_server s, uint64_t id, const int L[4], const double* links, double eps, int n_steps) {
    if (!s || !L || !links || !(eps > 0.0) || n_steps < 1) return fail(QCB_EINVAL, "serve submit: invalid argument");
    int64_t V = 0;
    if (!lattice_ok(L, &V)) return fail(QCB_EINVAL, "serve submit: extents must be even, >= 2, volume <= 2^30");
    Request* r = new (std::nothrow) Request();
    if (!r) return fail(QCB_ENOMEM, "host allocation");
    r->id = id;
    r->g = make_geom(L);
    r->eps = eps;
    r->n_steps = n_steps;
    r->input.assign(links, links + (size_t)V * 72);
    const size_t lb = align256(link_bytes(s->fmt, r->g.Vh));
    r->off_out = lb;
    r->off_z = 2 * lb;
    r->off_meas = 2 * lb + align256(alg_bytes(s->fmt, r->g.Vh));
    r->bytes = r->off_meas + align256((size_t)n_steps * 3 * sizeof(double));
    if (QCB_SERVE_FUSED_MEAS && !is_big(r)) {
        r->off_halves = r->bytes;
        r->bytes += align256(halves_bytes(s->fmt, r->g.Vh));
    }
    if (r->bytes > s->budget) {
        const size_t need = r->bytes;
        delete r;
        return fail(QCB_ENOMEM, "serve submit: request needs %zu bytes, budget is %zu", need, s->budget);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->err != QCB_OK) {
            delete r;
            return fail(s->err, "server stopped: %s", s->errmsg.c_str());
        }
        r->t_submit = s->now();
        s->pending.push_back(r);
        s->submitted++;
    }
    s->cv_work.notify_one();
    return QCB_OK;
}

// Pops one completed request: returns 1 (and fills the outputs) or 0 if none is ready.
// tQE must hold 3 * max_steps doubles; times are seconds on the server's clock.
int qcb_serve_poll(qcb_server s, uint64_t* id, double* tQE, int max_steps, int* n_steps, double* times) {
    if (!s) return fail(QCB_EINVAL, "null server");
    Request* r = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->done.empty()) return s->err != QCB_OK ? fail(s->err, "server: %s", s->errmsg.c_str()) : 0;
        r = s->done.front();
        s->done.pop_front();
    }
    if (id) *id = r->id;
    if (n_steps) *n_steps = r->n_steps;
    if (tQE) memcpy(tQE, r->tqe.data(), sizeof(double) * 3 * std::min(max_steps, r->n_steps));
    if (times) {
        times[0] = r->t_submit;
        times[1] = r->t_admit;
        times[2] = r->t_done;
    }
    delete r;
    return 1;
}

// Waits (bounded) until every submitted request has completed.
int qcb_serve_wait(qcb_server s, double timeout_s) {
    if (!s) return fail(QCB_EINVAL, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                        [&] { return s->completed == s->submitted || s->err != QCB_OK; });
    if (s->err != QCB_OK) return fail(s->err, "server: %s", s->errmsg.c_str());
    if (!ok) return fail(QCB_ETIMEOUT, "serve wait: %llu of %llu requests done", (unsigned long long)s->completed,
                         (unsigned long long)s->submitted);
    return QCB_OK;
}

// stats: [0] submitted, [1] completed, [2] scheduler ticks, [3] peak resident requests,
// [4] peak bytes in use, [5] bytes in use, [6] scheduler busy seconds, [7] queued requests.
int qcb_serve_stats(qcb_server s, double* out) {
    if (!s || !out) return fail(QCB_EINVAL, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out[0] = (double)s->submitted;
    out[1] = (double)s->completed;
    out[2] = (double)s->ticks;
    out[3] = (double)s->active_peak;
    out[4] = (double)s->bytes_peak;
    out[5] = (double)s->bytes_in_use;
    out[6] = s->busy;
    out[7] = (double)s->pending.size();
    return QCB_OK;
}

}  // extern "C"
