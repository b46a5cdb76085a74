// qcb_api.cu -- C ABI of libqcb.so: handles, launches and reductions.
//
// One handle = one periodic lattice resident on one GPU (the reference's GaugeField +
// GeometryCB on one MPI rank with a periodic halo, src/gauge/GaugeField.h:18-62).
// Kernels are launched on the handle's stream; results return to the host only from
// calls that produce host values.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <new>
#include <string>

#include "qcb_internal.h"
#include "qcb_ops.h"

// Measured flows take each measurement from the following RK3 step's stage 1 (clover halves) rather
// than a separate clover pass; 0 keeps the clover pass for every measurement.
#ifndef QCB_FLOW_FUSED_MEAS
#define QCB_FLOW_FUSED_MEAS 1
#endif

using namespace qcb;

// ====================================================================== errors
namespace {
thread_local std::string g_err;
std::atomic<uint64_t> g_launches{0};
int g_sm_count = 0;
}  // namespace

int qcb::sm_count() {
    if (g_sm_count == 0) {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
        g_sm_count = n;
    }
    return g_sm_count;
}

void qcb::note_launches(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

int qcb::fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) return fail(QCB_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)
#define RET(call)                    \
    do {                             \
        int r_ = (call);             \
        if (r_ != QCB_OK) return r_; \
    } while (0)

namespace {

inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }
// Grid size of the grid-stride reduction kernels: bounded so that the partial vectors
// stay small, a multiple of the 148 SMs of a B200.
inline unsigned red_blocks(int64_t n, int threads) {
    unsigned b = blocks_for(n, threads);
    return b < 148u * 8u ? b : 148u * 8u;
}

cudaEvent_t get_event(qcb_field_s* f) {
    if (!f->event_pool.empty()) {
        cudaEvent_t e = f->event_pool.back();
        f->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Launch wrapper: launch counting, error check and optional event timing on the stream.
template <class Fn>
int launch(qcb_field_s* f, int kclass, Fn&& fn) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (f->timing) {
        a = get_event(f);
        b = get_event(f);
        CK(cudaEventRecord(a, f->stream));
    }
    cudaError_t e = fn();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return fail(QCB_ECUDA, "kernel launch: %s", cudaGetErrorString(e));
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (f->timing) {
        CK(cudaEventRecord(b, f->stream));
        f->pending.push_back(TimedLaunch{kclass, a, b});
    }
    return QCB_OK;
}

int ensure_partials(qcb_field_s* f, size_t n) {
    if (f->partials_cap >= n) return QCB_OK;
    if (f->partials) cudaFree(f->partials);
    f->partials = nullptr;
    f->partials_cap = 0;
    CK(cudaMalloc(&f->partials, n * sizeof(double)));
    f->partials_cap = n;
    return QCB_OK;
}
int ensure_staging(qcb_field_s* f) {
    if (f->staging) return QCB_OK;
    CK(cudaMalloc(&f->staging, (size_t)f->g.V * 36 * sizeof(double2)));
    return QCB_OK;
}
// The staging buffer for a use on the field's stream; refused while a prefetched configuration
// occupies it.
int staging_acquire(qcb_field_s* f) {
    if (f->prefetch_pending)
        return fail(QCB_EINVAL, "a prefetched configuration occupies the staging buffer: commit it first");
    return ensure_staging(f);
}
// Marks the end of the staging buffer's latest use on the field's stream: the next prefetch copy
// waits for this point only, not for everything queued on the stream after it.
int staging_release(qcb_field_s* f) {
    if (!f->ev_staging) CK(cudaEventCreateWithFlags(&f->ev_staging, cudaEventDisableTiming));
    CK(cudaEventRecord(f->ev_staging, f->stream));
    f->staging_used = true;
    return QCB_OK;
}
int ensure_alt(qcb_field_s* f) {
    if (f->alt) return QCB_OK;
    CK(cudaMalloc(&f->alt, link_bytes(f->fmt, f->g.Vh)));
    return QCB_OK;
}

int check_err_flag(qcb_field_s* f) {
    int h = 0;
    CK(cudaMemcpyAsync(&h, f->d_err, sizeof(int), cudaMemcpyDeviceToHost, f->stream));
    CK(cudaStreamSynchronize(f->stream));
    if (h) {
        CK(cudaMemsetAsync(f->d_err, 0, sizeof(int), f->stream));
        if (h & DERR_BULK_WAIT)
            return fail(QCB_ETIMEOUT, "heatbath: bulk copy of the block's links did not complete (links left unchanged)");
        if (h & DERR_KP_SCALE)
            return fail(QCB_ERANGE, "heatbath: zero or non-finite SU(2) projection of the staple (link left unchanged)");
        return fail(QCB_ERANGE, "heatbath: Kennedy-Pendleton attempt cap (2^20) reached (link left unchanged)");
    }
    return QCB_OK;
}

// reduction of nb partial vectors of nv doubles into dst (device)
int finalize(qcb_field_s* f, int nb, int nv, unsigned max_mask, double* dst) {
    return launch(f, QCB_K_OTHER, [&] {
        k_finalize<<<1, 256, 0, f->stream>>>(f->partials, nb, nv, max_mask, dst);
        return cudaGetLastError();
    });
}

// --- enqueue helpers (no host synchronisation) --------------------------------------
int enq_plaquette(qcb_field_s* f, double* dst) {
    const unsigned nbx = red_blocks(f->g.Vh, 256);
    RET(ensure_partials(f, (size_t)nbx * 2));
    RET(launch(f, QCB_K_PLAQ, [&] { return fmt_ops(f->fmt).plaquette(f->g, f->links, f->partials, nbx, f->stream); }));
    return finalize(f, (int)(nbx * 2), 1, 0u, dst);
}
// Clover sums (q, e, plaquette) -> dst[0..2]; the plaquette sum comes from leaf 1 of each plane.
// One block per 128 half-sites (up to the grid's y limit): the blocks run in site order, so the
// pass sweeps the lattice once in t and a link's neighbours are still in L2 when the front reaches
// them (a capped grid-stride loop jumps across the lattice and re-reads them from DRAM).
int enq_clover(qcb_field_s* f, double* dst) {
    const unsigned nbx = clover_blocks(f->g.Vh);
    RET(ensure_partials(f, (size_t)nbx * 6 * 3));
    RET(launch(f, QCB_K_CLOVER, [&] { return fmt_ops(f->fmt).clover(f->g, f->links, f->partials, nbx, f->stream); }));
    return finalize(f, (int)(nbx * 6), 3, 0u, dst);
}

int read_results(qcb_field_s* f, int n) {
    CK(cudaMemcpyAsync(f->h_res, f->d_res, n * sizeof(double), cudaMemcpyDeviceToHost, f->stream));
    CK(cudaStreamSynchronize(f->stream));
    return QCB_OK;
}

int upload_from_staging(qcb_field_s* f, int bswap) {
    return launch(f, QCB_K_OTHER,
                  [&] { return fmt_ops(f->fmt).aos_to_soa(f->g, f->staging, f->links, bswap, f->stream); });
}
int download_to_staging(qcb_field_s* f, int bswap) {
    return launch(f, QCB_K_OTHER,
                  [&] { return fmt_ops(f->fmt).soa_to_aos(f->g, f->links, f->staging, bswap, f->stream); });
}

// One RK3 step on the flow's field: stage 1 reads links and writes alt, stage 2 the reverse,
// stage 3 links -> alt again; the buffers then swap so that links holds the result.
int flow_step(qcb_flow_s* fl) {
    qcb_field_s* f = fl->fld;
    RET(ensure_alt(f));
    const int rep = needs_reproject(f->prec, f->store);
    for (int stage = 1; stage <= 3; stage++) {
        void* win = (stage == 2) ? f->alt : f->links;
        void* wout = (stage == 2) ? f->links : f->alt;
        RET(launch(f, QCB_K_FLOW,
                   [&] { return fmt_ops(f->fmt).flow1(f->g, win, wout, fl->z, fl->eps, stage, rep, f->stream); }));
    }
    void* t = f->links;
    f->links = f->alt;
    f->alt = t;
    return QCB_OK;
}

// One RK3 step that also measures its input configuration: stage 1 writes the clover halves
// (k_flow_stage1_meas; its links are those of the plain stage 1), their per-site sum gives
// (q, e, plaquette sum) in dst[0..2], then stages 2 and 3 as in flow_step.  The standalone clover
// pass forms every leaf with three products a plane and site; here the force's own staples give
// the clover with two products a plane and link.
int flow_step_meas(qcb_flow_s* fl, double* dst) {
    qcb_field_s* f = fl->fld;
    RET(ensure_alt(f));
    const int rep = needs_reproject(f->prec, f->store);
    RET(launch(f, QCB_K_FLOW, [&] {
        return fmt_ops(f->fmt).flow1_meas(f->g, f->links, f->alt, fl->z, fl->eps, rep, fl->halves, f->stream);
    }));
    const unsigned nb = halves_blocks(f->g.Vh);
    RET(launch(f, QCB_K_CLOVER,
               [&] { return fmt_ops(f->fmt).clover_halves(f->g, fl->halves, f->partials, nb, f->stream); }));
    RET(finalize(f, (int)nb, 3, 0u, dst));
    for (int stage = 2; stage <= 3; stage++) {
        void* win = (stage == 2) ? f->alt : f->links;
        void* wout = (stage == 2) ? f->links : f->alt;
        RET(launch(f, QCB_K_FLOW,
                   [&] { return fmt_ops(f->fmt).flow1(f->g, win, wout, fl->z, fl->eps, stage, rep, f->stream); }));
    }
    void* t = f->links;
    f->links = f->alt;
    f->alt = t;
    return QCB_OK;
}

// The measurement of the flowed field alone through the measuring stage 1 (its stage-1 output, in
// the spare buffer, is left unused): the last measurement of a run, so that every row of a measured
// flow comes from the same arithmetic.
int meas_halves_only(qcb_flow_s* fl, double* dst) {
    qcb_field_s* f = fl->fld;
    RET(ensure_alt(f));
    const int rep = needs_reproject(f->prec, f->store);
    RET(launch(f, QCB_K_CLOVER, [&] {
        return fmt_ops(f->fmt).flow1_meas(f->g, f->links, f->alt, fl->z, fl->eps, rep, fl->halves, f->stream);
    }));
    const unsigned nb = halves_blocks(f->g.Vh);
    RET(launch(f, QCB_K_CLOVER,
               [&] { return fmt_ops(f->fmt).clover_halves(f->g, fl->halves, f->partials, nb, f->stream); }));
    return finalize(f, (int)nb, 3, 0u, dst);
}

// ------------------------------------------------------------------ flow step graphs
// Without per-launch timing, the flow's repeated launch sequences are captured once as CUDA graphs
// and replayed: two RK3 steps (six stage launches; the ping-pong buffers are back in place after
// them), and one measurement block of qcb_flow_measure (clover pass into a fixed slot, the row
// scatter, then n_rk RK3 steps).  Replays launch the same kernels with the same arguments as the
// plain launches, so results are identical bit for bit.
constexpr int kMeasSlot = 32;  // d_res offset of the measurement slot (q, e, plaquette sums)

int meas_block(qcb_flow_s* fl, int n_rk);
__global__ void k_meas_scatter(const double* slot, double* meas, int* counter);
// Graphs need a capturable stream: not the legacy default stream, and no per-launch timing events.
bool graphs_ok(const qcb_field_s* f) { return !f->timing && f->stream != nullptr; }

int flow_graph_body(qcb_flow_s* fl, int kind, int n_rk) {
    if (kind == 1) {
        RET(flow_step(fl));
        return flow_step(fl);
    }
    return meas_block(fl, n_rk);
}

// Runs the body of graph `kind` once: replays a cached graph captured from the same buffers, or
// captures one (the capture moves the host's ping-pong pointers as the body does; the graph is then
// launched once to do the work).
int flow_graph_run(qcb_flow_s* fl, int kind, int n_rk) {
    qcb_field_s* f = fl->fld;
    const void* links0 = f->links;
    FlowGraph* hit = nullptr;
    for (auto& g : fl->graphs)
        if (g.exec && g.kind == kind && g.n_rk == n_rk && g.links == links0 && g.partials == f->partials &&
            g.meas == fl->d_meas)
            hit = &g;
    if (!hit) {
        FlowGraph* slot = &fl->graphs[0];
        for (auto& g : fl->graphs)
            if (!g.exec || g.last_use < slot->last_use) slot = &g;
        if (slot->exec) cudaGraphExecDestroy(slot->exec);
        *slot = FlowGraph{};
        const uint64_t n0 = g_launches.load();
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(f->stream, cudaStreamCaptureModeThreadLocal));
        int r = flow_graph_body(fl, kind, n_rk);
        const cudaError_t e = cudaStreamEndCapture(f->stream, &graph);
        const int kernels = (int)(g_launches.load() - n0);
        g_launches.fetch_sub((uint64_t)kernels);  // counted when a replay runs them
        if (r != QCB_OK) {
            if (graph) cudaGraphDestroy(graph);
            return r;
        }
        if (e != cudaSuccess) return fail(QCB_ECUDA, "flow graph capture: %s", cudaGetErrorString(e));
        const cudaError_t ei = cudaGraphInstantiate(&slot->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            slot->exec = nullptr;
            return fail(QCB_ECUDA, "flow graph instantiate: %s", cudaGetErrorString(ei));
        }
        slot->kind = kind;
        slot->n_rk = n_rk;
        slot->kernels = kernels;
        slot->links = links0;
        slot->partials = f->partials;
        slot->meas = fl->d_meas;
        hit = slot;
        // the capture left the host pointers where the body leaves them; the replay below is the
        // body's one execution, from the buffers it was captured from
        if (f->links != links0) {
            void* t = f->links;
            f->links = f->alt;
            f->alt = t;
        }
    }
    hit->last_use = ++fl->graph_clock;
    CK(cudaGraphLaunch(hit->exec, f->stream));
    g_launches.fetch_add((uint64_t)hit->kernels);
    // the body swaps the ping-pong buffers once per RK3 step
    const int steps = kind == 1 ? 2 : n_rk;
    if (steps & 1) {
        void* t = f->links;
        f->links = f->alt;
        f->alt = t;
    }
    return QCB_OK;
}

// One measurement of the flowed field -- (q, e and the plaquette sum) into the fixed slot, copied to
// the next row of the measurement buffer -- followed by n_rk RK3 steps.  With the halves buffer in
// place (measured flows with RK3 steps) the measurement comes from the measuring stage 1: that of
// the following step, or for the last measurement one whose output is left unused.
int meas_block(qcb_flow_s* fl, int n_rk) {
    qcb_field_s* f = fl->fld;
    double* slot = f->d_res + kMeasSlot;
    const bool fused = n_rk > 0 && fl->halves;
    if (fused)
        RET(flow_step_meas(fl, slot));
    else if (fl->halves)
        RET(meas_halves_only(fl, slot));
    else
        RET(enq_clover(f, slot));
    RET(launch(f, QCB_K_OTHER, [&] {
        k_meas_scatter<<<1, 1, 0, f->stream>>>(slot, fl->d_meas, fl->d_count);
        return cudaGetLastError();
    }));
    for (int k = fused ? 1 : 0; k < n_rk; k++) RET(flow_step(fl));
    return QCB_OK;
}

void drop_flow_graphs(qcb_flow_s* fl) {
    for (auto& g : fl->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = FlowGraph{};
    }
}

bool valid_L(const int L[4]) { return L && lattice_ok(L); }

int field_new(const int L[4], int prec, int store, cudaStream_t stream, qcb_field_s** out) {
    if (!out) return fail(QCB_EINVAL, "null output handle");
    if (!valid_L(L)) return fail(QCB_EINVAL, "lattice extents must be even, >= 2, volume <= 2^30");
    if (prec != QCB_PREC_F64 && prec != QCB_PREC_F32) return fail(QCB_EINVAL, "prec must be 64 or 32");
    if (store != QCB_STORE_18 && store != QCB_STORE_12) return fail(QCB_EINVAL, "store must be 0 (18) or 1 (12)");
    qcb_field_s* f = new (std::nothrow) qcb_field_s();
    if (!f) return fail(QCB_ENOMEM, "host allocation");
    for (int d = 0; d < 4; d++) f->L[d] = L[d];
    f->g = make_geom(L);
    f->prec = prec;
    f->store = store;
    f->fmt = fmt_of(prec, store);
    cudaGetDevice(&f->device);
    int r = QCB_OK;
    cudaError_t e;
    if (stream) {
        f->stream = stream;
    } else {
        e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete f;
            return fail(QCB_ECUDA, "stream: %s", cudaGetErrorString(e));
        }
        f->own_stream = true;
    }
    e = cudaMalloc(&f->links, link_bytes(f->fmt, f->g.Vh));
    if (e == cudaSuccess) e = cudaMalloc(&f->d_res, 64 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&f->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&f->h_res, 64 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemsetAsync(f->d_err, 0, sizeof(int), f->stream);
    if (e != cudaSuccess) {
        r = fail(e == cudaErrorMemoryAllocation ? QCB_ENOMEM : QCB_ECUDA, "field allocation: %s",
                 cudaGetErrorString(e));
        qcb_field_destroy(f);
        return r;
    }
    *out = f;
    return qcb_cold_start(f);
}

}  // namespace

// Deterministic final reduction (one block, fixed summation order for a given nb).
__global__ void qcb::k_finalize(const double* partials, int nb, int nv, unsigned max_mask, double* out) {
    __shared__ double sm[256];
    for (int k = 0; k < nv; k++) {
        const bool ismax = (max_mask >> k) & 1u;
        double acc = 0.0;
        for (int i = threadIdx.x; i < nb; i += 256) {
            double v = partials[(size_t)i * nv + k];
            acc = ismax ? fmax(acc, v) : acc + v;
        }
        sm[threadIdx.x] = acc;
        __syncthreads();
        for (int s = 128; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) sm[threadIdx.x] = ismax ? fmax(sm[threadIdx.x], sm[threadIdx.x + s])
                                                              : sm[threadIdx.x] + sm[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[k] = sm[0];
        __syncthreads();
    }
}

// Per-lattice deterministic sums of tile partials (one block per lattice, fixed order).
__global__ void qcb::k_lat_finalize(const LatDesc* __restrict__ lats, const LatDesc one,
                                    const double* __restrict__ partials, int m, int nv, int scale_mode, double* out) {
    __shared__ double sm[256];
    const LatDesc* d = lats ? lats + blockIdx.x : &one;
    const int t0 = m * d->nb_begin, nt = m * d->nb;
    for (int k = 0; k < nv; k++) {
        double acc = 0.0;
        for (int i = threadIdx.x; i < nt; i += 256) acc += partials[(size_t)(t0 + i) * nv + k];
        sm[threadIdx.x] = acc;
        __syncthreads();
        for (int s = 128; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            double v = sm[0];
            if (scale_mode == 1) v /= 6.0 * (double)d->g.V;
            if (scale_mode == 2 && k == 1) v /= (double)d->g.V;
            out[(size_t)blockIdx.x * nv + k] = v;
        }
        __syncthreads();
    }
}

namespace {
__global__ void k_diag_exp(const double2* Z, int n, double coeff, int f32, double2* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    M3<double> z;
    for (int e = 0; e < 9; e++) z.e[e] = mkc(Z[i * 9 + e].x, Z[i * 9 + e].y);
    for (int e = 0; e < 9; e++) z.e[e] = scl(coeff, z.e[e]);
    M3<double> r;
    if (f32) {
        r = convert<double>(exp_su3(convert<float>(z)));
    } else {
        r = exp_su3(z);
    }
    for (int e = 0; e < 9; e++) out[i * 9 + e] = make_double2(r.e[e].re, r.e[e].im);
}
// Fused multiply-add throughput probe: 8 independent chains per thread, unrolled, so that the FMA
// pipe rather than latency sets the rate; the result is kept live through a data-dependent store.
template <typename T>
__global__ void __launch_bounds__(256) k_fma_rate(T a, T b, int iters, T* out) {
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = (T)(threadIdx.x + k) * (T)1e-3;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == (T)-1) out[0] = s;  // never true for these inputs; keeps the chains
}

// Copies one measurement (q, e, plaquette sums) from the fixed slot the clover pass wrote into row
// *counter of the measurement buffer and advances the counter (one thread; the host sizes the buffer
// for every row it launches).
__global__ void k_meas_scatter(const double* slot, double* meas, int* counter) {
    const int c = *counter;
    meas[3 * c] = slot[0];
    meas[3 * c + 1] = slot[1];
    meas[3 * c + 2] = slot[2];
    *counter = c + 1;
}
__global__ void k_diag_philox(uint4 ctr, uint2 key, int n, uint4* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t c[4] = {ctr.x + (uint32_t)i, ctr.y, ctr.z, ctr.w};
    philox4x32_10(c, key.x, key.y);
    out[i] = make_uint4(c[0], c[1], c[2], c[3]);
}
}  // namespace

int qcb::field_upload_host(qcb_field_s* f, const double* host, int bswap) {
    RET(staging_acquire(f));
    CK(cudaMemcpyAsync(f->staging, host, (size_t)f->g.V * 36 * sizeof(double2), cudaMemcpyHostToDevice, f->stream));
    RET(upload_from_staging(f, bswap));
    RET(staging_release(f));
    CK(cudaStreamSynchronize(f->stream));
    return QCB_OK;
}
int qcb::field_download_host(qcb_field_s* f, double* host, int bswap) {
    RET(staging_acquire(f));
    RET(download_to_staging(f, bswap));
    CK(cudaMemcpyAsync(host, f->staging, (size_t)f->g.V * 36 * sizeof(double2), cudaMemcpyDeviceToHost, f->stream));
    RET(staging_release(f));
    CK(cudaStreamSynchronize(f->stream));
    return QCB_OK;
}

#ifdef QCB_CHECKED
// Every translation unit of the checked build registers the reader of its out-of-bounds record.
namespace qcb {
static std::vector<OobTake>& oob_registry() {
    static std::vector<OobTake> v;
    return v;
}
void register_oob(OobTake fn) { oob_registry().push_back(fn); }
}  // namespace qcb
#endif

// ====================================================================== C ABI
extern "C" {

const char* qcb_last_error(void) { return g_err.c_str(); }
#ifdef QCB_CHECKED
const char* qcb_version(void) { return "qcb 0.1 (sm_100a, checked)"; }
#else
const char* qcb_version(void) { return "qcb 0.1 (sm_100a)"; }
#endif

int qcb_debug_oob(int* checked, uint64_t* count, uint64_t* first) {
    if (!checked || !count || !first) return fail(QCB_EINVAL, "null argument");
    *count = 0;
    *first = 0;
#ifdef QCB_CHECKED
    *checked = 1;
    CK(cudaDeviceSynchronize());
    for (OobTake fn : oob_registry()) {
        unsigned long long c = 0, f0 = 0;
        const cudaError_t e = fn(&c, &f0);
        if (e == cudaErrorInvalidSymbol) {  // a unit without device code keeps no record
            cudaGetLastError();
            continue;
        }
        CK(e);
        if (c && !*count) *first = f0;
        *count += c;
    }
#else
    *checked = 0;
#endif
    return QCB_OK;
}

int qcb_debug_probe_link(qcb_field f, int mu, int parity, int64_t h) {
    if (!f) return fail(QCB_EINVAL, "null field");
#ifndef QCB_CHECKED
    // only the checked build may send an index outside the field to the device, where its own
    // check catches it
    if (mu < 0 || mu > 3 || parity < 0 || parity > 1 || h < 0 || h >= f->g.Vh)
        return fail(QCB_EINVAL, "probe: (mu, parity, h) outside the field");
#endif
    if (h < INT32_MIN || h > INT32_MAX) return fail(QCB_EINVAL, "probe: h outside the int range");
    return launch(f, QCB_K_OTHER, [&] {
        return fmt_ops(f->fmt).probe_link(f->g, f->links, mu, parity, (int)h, f->d_res, f->stream);
    });
}
uint64_t qcb_launch_count(void) { return g_launches.load(); }

int qcb_field_create(const int L[4], int prec, int store, qcb_field* out) {
    return field_new(L, prec, store, nullptr, out);
}

int qcb_field_destroy(qcb_field f) {
    if (!f) return QCB_OK;
    if (f->stream) cudaStreamSynchronize(f->stream);
    for (auto& t : f->pending) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (auto e : f->event_pool) cudaEventDestroy(e);
    if (f->copy_stream) {
        cudaStreamSynchronize(f->copy_stream);
        cudaStreamDestroy(f->copy_stream);
    }
    if (f->ev_copied) cudaEventDestroy(f->ev_copied);
    if (f->ev_staging) cudaEventDestroy(f->ev_staging);
    if (f->links) cudaFree(f->links);
    if (f->alt) cudaFree(f->alt);
    if (f->staging) cudaFree(f->staging);
    if (f->partials) cudaFree(f->partials);
    if (f->d_res) cudaFree(f->d_res);
    if (f->d_err) cudaFree(f->d_err);
    if (f->h_res) cudaFreeHost(f->h_res);
    if (f->own_stream && f->stream) cudaStreamDestroy(f->stream);
    delete f;
    return QCB_OK;
}

int qcb_field_info(qcb_field f, int L[4], int* prec, int* store, size_t* device_bytes) {
    if (!f) return fail(QCB_EINVAL, "null field");
    if (L)
        for (int d = 0; d < 4; d++) L[d] = f->L[d];
    if (prec) *prec = f->prec;
    if (store) *store = f->store;
    if (device_bytes) *device_bytes = link_bytes(f->fmt, f->g.Vh);
    return QCB_OK;
}

void* qcb_field_stream(qcb_field f) { return f ? (void*)f->stream : nullptr; }

int qcb_field_set_stream(qcb_field f, void* s) {
    if (!f) return fail(QCB_EINVAL, "null field");
    CK(cudaStreamSynchronize(f->stream));
    if (f->own_stream) cudaStreamDestroy(f->stream);
    f->own_stream = false;
    f->stream = (cudaStream_t)s;
    return QCB_OK;
}

int qcb_field_sync(qcb_field f) {
    if (!f) return fail(QCB_EINVAL, "null field");
    CK(cudaStreamSynchronize(f->stream));
    return QCB_OK;
}

int qcb_field_upload_aos(qcb_field f, const double* links) {
    if (!f || !links) return fail(QCB_EINVAL, "null argument");
    return field_upload_host(f, links, 0);
}
int qcb_field_prefetch_aos(qcb_field f, const double* links) {
    if (!f || !links) return fail(QCB_EINVAL, "null argument");
    if (f->prefetch_pending) return fail(QCB_EINVAL, "a prefetched configuration is pending: commit it first");
    RET(ensure_staging(f));
    if (!f->copy_stream) {
        CK(cudaStreamCreateWithFlags(&f->copy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&f->ev_copied, cudaEventDisableTiming));
    }
    if (f->staging_used) CK(cudaStreamWaitEvent(f->copy_stream, f->ev_staging, 0));
    CK(cudaMemcpyAsync(f->staging, links, (size_t)f->g.V * 36 * sizeof(double2), cudaMemcpyHostToDevice,
                       f->copy_stream));
    CK(cudaEventRecord(f->ev_copied, f->copy_stream));
    f->prefetch_pending = true;
    return QCB_OK;
}
int qcb_field_commit_prefetch(qcb_field f) {
    if (!f) return fail(QCB_EINVAL, "null field");
    if (!f->prefetch_pending) return fail(QCB_EINVAL, "no prefetched configuration to commit");
    CK(cudaStreamWaitEvent(f->stream, f->ev_copied, 0));
    f->prefetch_pending = false;
    RET(upload_from_staging(f, 0));
    return staging_release(f);
}
int qcb_field_download_aos(qcb_field f, double* links) {
    if (!f || !links) return fail(QCB_EINVAL, "null argument");
    return field_download_host(f, links, 0);
}
int qcb_field_upload_aos_device(qcb_field f, const double* d_links) {
    if (!f || !d_links) return fail(QCB_EINVAL, "null argument");
    return launch(f, QCB_K_OTHER,
                  [&] { return fmt_ops(f->fmt).aos_to_soa(f->g, (const double2*)d_links, f->links, 0, f->stream); });
}
int qcb_field_download_aos_device(qcb_field f, double* d_links) {
    if (!f || !d_links) return fail(QCB_EINVAL, "null argument");
    return launch(f, QCB_K_OTHER,
                  [&] { return fmt_ops(f->fmt).soa_to_aos(f->g, f->links, (double2*)d_links, 0, f->stream); });
}

int qcb_field_copy(qcb_field dst, qcb_field src) {
    if (!dst || !src) return fail(QCB_EINVAL, "null field");
    for (int d = 0; d < 4; d++)
        if (dst->L[d] != src->L[d]) return fail(QCB_EINVAL, "copy between different lattices");
    if (dst == src) return QCB_OK;
    if (dst->stream != src->stream) {
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CK(cudaEventRecord(ev, src->stream));
        CK(cudaStreamWaitEvent(dst->stream, ev, 0));
        cudaEventDestroy(ev);
    }
    if (dst->fmt == src->fmt) {
        CK(cudaMemcpyAsync(dst->links, src->links, link_bytes(dst->fmt, dst->g.Vh), cudaMemcpyDeviceToDevice,
                           dst->stream));
    } else {
        RET(staging_acquire(dst));
        RET(launch(dst, QCB_K_OTHER,
                   [&] { return fmt_ops(src->fmt).soa_to_aos(src->g, src->links, dst->staging, 0, dst->stream); }));
        RET(upload_from_staging(dst, 0));
        RET(staging_release(dst));
    }
    // src's later work (a heatbath, an upload) must not overwrite src's links while dst's stream is
    // still reading them: src's stream waits for the end of the copy.
    if (dst->stream != src->stream) {
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        CK(cudaEventRecord(ev, dst->stream));
        CK(cudaStreamWaitEvent(src->stream, ev, 0));
        cudaEventDestroy(ev);
    }
    return QCB_OK;
}

int qcb_cold_start(qcb_field f) {
    if (!f) return fail(QCB_EINVAL, "null field");
    return launch(f, QCB_K_OTHER, [&] { return fmt_ops(f->fmt).start(f->g, f->links, 0, 0ull, f->stream); });
}

int qcb_hot_start(qcb_field f, uint64_t seed) {
    if (!f) return fail(QCB_EINVAL, "null field");
    return launch(f, QCB_K_OTHER, [&] { return fmt_ops(f->fmt).start(f->g, f->links, 1, seed, f->stream); });
}

int qcb_reunitarize(qcb_field f) {
    if (!f) return fail(QCB_EINVAL, "null field");
    return launch(f, QCB_K_OTHER, [&] { return fmt_ops(f->fmt).reunitarize(f->g, f->links, f->stream); });
}

int qcb_unitarity(qcb_field f, double* max_err, double* mean_err) {
    if (!f) return fail(QCB_EINVAL, "null field");
    const unsigned nbx = red_blocks(f->g.Vh, 256);
    RET(ensure_partials(f, (size_t)nbx * 8 * 2));
    RET(launch(f, QCB_K_OTHER,
               [&] { return fmt_ops(f->fmt).unitarity(f->g, f->links, f->partials, nbx, f->stream); }));
    RET(finalize(f, (int)(nbx * 8), 2, 1u, f->d_res));
    RET(read_results(f, 2));
    if (max_err) *max_err = f->h_res[0];
    if (mean_err) *mean_err = f->h_res[1] / (4.0 * (double)f->g.V);
    return QCB_OK;
}

int qcb_shift(qcb_field f, const int s[4]) {
    if (!f || !s) return fail(QCB_EINVAL, "null argument");
    int sm[4];
    bool any = false;
    for (int d = 0; d < 4; d++) {
        sm[d] = ((s[d] % f->L[d]) + f->L[d]) % f->L[d];
        any = any || sm[d] != 0;
    }
    if (!any) return QCB_OK;
    RET(ensure_alt(f));
    RET(launch(f, QCB_K_OTHER, [&] { return fmt_ops(f->fmt).shift(f->g, f->links, f->alt, sm, f->stream); }));
    void* t = f->links;
    f->links = f->alt;
    f->alt = t;
    return QCB_OK;
}

int qcb_random_shift(qcb_field f, uint64_t seed, uint64_t idx, int max_shift, int s_out[4]) {
    if (!f) return fail(QCB_EINVAL, "null field");
    uint32_t c[4] = {0u, (uint32_t)idx, (uint32_t)(idx >> 32), TAG_SHIFT};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    int s[4];
    for (int d = 0; d < 4; d++) {
        uint32_t n = (uint32_t)(max_shift > 0 ? max_shift : f->L[d]);
        s[d] = (int)(((uint64_t)c[d] * n) >> 32);
        if (s_out) s_out[d] = s[d];
    }
    return qcb_shift(f, s);
}

int qcb_hb_subsweep(qcb_field f, double beta, int n_hits, uint64_t seed, uint32_t sweep, int parity, int mu) {
    if (!f) return fail(QCB_EINVAL, "null field");
    if (parity < 0 || parity > 1 || mu < 0 || mu > 3 || n_hits < 0 || !(beta > 0.0))
        return fail(QCB_EINVAL, "heatbath: parity in {0,1}, mu in 0..3, n_hits >= 0, beta > 0");
    const int rep = needs_reproject(f->prec, f->store);
    return launch(f, QCB_K_HB, [&] {
        return fmt_ops(f->fmt).hb1(f->g, f->links, parity, mu, -0.75 / beta, n_hits, seed, sweep, rep, f->d_err,
                                   f->stream);
    });
}

int qcb_hb_link(qcb_field f, int64_t site, int mu, double beta, int n_hits, uint64_t seed, uint32_t sweep,
                double* A_out) {
    if (!f) return fail(QCB_EINVAL, "null field");
    if (site < 0 || site >= f->g.V || mu < 0 || mu > 3 || n_hits < 0 || !(beta > 0.0))
        return fail(QCB_EINVAL, "heatbath link: site in [0, V), mu in 0..3, n_hits >= 0, beta > 0");
    int64_t r = site;
    int par = 0;
    for (int d = 0; d < 4; d++) {
        par += (int)(r % f->L[d]);
        r /= f->L[d];
    }
    par &= 1;
    const int rep = needs_reproject(f->prec, f->store);
    RET(launch(f, QCB_K_HB, [&] {
        return fmt_ops(f->fmt).hb_one(f->g, f->links, par, (int)(site >> 1), mu, -0.75 / beta, n_hits, seed, sweep,
                                      rep, f->d_err, (double2*)f->d_res, f->stream);
    }));
    RET(read_results(f, 18));
    if (A_out) memcpy(A_out, f->h_res, 18 * sizeof(double));
    return check_err_flag(f);
}

int qcb_hb_sweep(qcb_field f, double beta, int n_hits, uint64_t seed, uint32_t sweep) {
    for (int p = 0; p < 2; p++)
        for (int mu = 0; mu < 4; mu++) RET(qcb_hb_subsweep(f, beta, n_hits, seed, sweep, p, mu));
    return QCB_OK;
}

int qcb_plaquette(qcb_field f, double* plaq) {
    if (!f || !plaq) return fail(QCB_EINVAL, "null argument");
    RET(enq_plaquette(f, f->d_res));
    RET(read_results(f, 1));
    *plaq = f->h_res[0] / (6.0 * (double)f->g.V);
    return check_err_flag(f);
}

int qcb_clover_qe(qcb_field f, double* Q, double* E) {
    if (!f) return fail(QCB_EINVAL, "null field");
    RET(enq_clover(f, f->d_res));
    RET(read_results(f, 2));
    if (Q) *Q = f->h_res[0];
    if (E) *E = f->h_res[1] / (double)f->g.V;
    return QCB_OK;
}

// Lattice site (lexicographic index) -> (parity, half-site index); false outside the lattice.
static bool site_of(const qcb_field_s* f, int64_t site, int* par, int* h) {
    if (site < 0 || site >= f->g.V) return false;
    int64_t r = site;
    int p = 0;
    for (int d = 0; d < 4; d++) {
        p += (int)(r % f->L[d]);
        r /= f->L[d];
    }
    *par = p & 1;
    *h = (int)(site >> 1);
    return true;
}

int qcb_clover_site(qcb_field f, int64_t site, int mu, int nu, double* F_out) {
    int par = 0, h = 0;
    if (!f || !F_out || !site_of(f, site, &par, &h) || mu < 0 || mu > 3 || nu < 0 || nu > 3 || mu == nu)
        return fail(QCB_EINVAL, "clover site: site in [0, V), mu != nu in 0..3, non-null output");
    RET(launch(f, QCB_K_CLOVER, [&] {
        return fmt_ops(f->fmt).clover_site(f->g, f->links, par, h, mu, nu, f->d_res, f->stream);
    }));
    RET(read_results(f, 18));
    memcpy(F_out, f->h_res, 18 * sizeof(double));
    return QCB_OK;
}

int qcb_local_qe(qcb_field f, int64_t site, double* q, double* e) {
    int par = 0, h = 0;
    if (!f || !site_of(f, site, &par, &h)) return fail(QCB_EINVAL, "local q, e: site in [0, V)");
    RET(launch(f, QCB_K_CLOVER, [&] {
        return fmt_ops(f->fmt).clover_site(f->g, f->links, par, h, -1, -1, f->d_res, f->stream);
    }));
    RET(read_results(f, 2));
    if (q) *q = f->h_res[0];
    if (e) *e = f->h_res[1];
    return QCB_OK;
}

// ------------------------------------------------------------------ flow
int qcb_flow_create(qcb_field src, double eps, int prec, int store, qcb_flow* out) {
    if (!src || !out) return fail(QCB_EINVAL, "null argument");
    if (!(eps > 0.0)) return fail(QCB_EINVAL, "flow step must be > 0");
    qcb_flow_s* fl = new (std::nothrow) qcb_flow_s();
    if (!fl) return fail(QCB_ENOMEM, "host allocation");
    fl->eps = eps;
    // The flow owns its stream: it must outlive no other handle's resources.
    int r = field_new(src->L, prec, store, nullptr, &fl->fld);
    if (r != QCB_OK) {
        delete fl;
        return r;
    }
    cudaError_t e = cudaMalloc(&fl->z, alg_bytes(fl->fld->fmt, fl->fld->g.Vh));
    if (e == cudaSuccess) e = cudaMalloc(&fl->fld->alt, link_bytes(fl->fld->fmt, fl->fld->g.Vh));
    if (e != cudaSuccess) {
        r = fail(e == cudaErrorMemoryAllocation ? QCB_ENOMEM : QCB_ECUDA, "flow allocation: %s",
                 cudaGetErrorString(e));
        qcb_flow_destroy(fl);
        return r;
    }
    r = qcb_field_copy(fl->fld, src);
    if (r != QCB_OK) {
        qcb_flow_destroy(fl);
        return r;
    }
    *out = fl;
    return QCB_OK;
}

int qcb_flow_destroy(qcb_flow fl) {
    if (!fl) return QCB_OK;
    if (fl->fld && fl->fld->stream) cudaStreamSynchronize(fl->fld->stream);
    drop_flow_graphs(fl);
    if (fl->f1) cudaFree(fl->f1);
    if (fl->d_meas) cudaFree(fl->d_meas);
    if (fl->d_count) cudaFree(fl->d_count);
    if (fl->halves) cudaFree(fl->halves);
    if (fl->z) cudaFree(fl->z);
    qcb_field_destroy(fl->fld);
    delete fl;
    return QCB_OK;
}

int qcb_flow_copy(qcb_flow fl, qcb_field src) {
    if (!fl || !src) return fail(QCB_EINVAL, "null argument");
    return qcb_field_copy(fl->fld, src);
}

int qcb_flow_rk3(qcb_flow fl, int n) {
    if (!fl || n < 0) return fail(QCB_EINVAL, "invalid argument");
    if (graphs_ok(fl->fld) && n >= 2) {
        RET(ensure_alt(fl->fld));
        for (; n >= 2; n -= 2) RET(flow_graph_run(fl, 1, 0));
    }
    for (int i = 0; i < n; i++) RET(flow_step(fl));
    return QCB_OK;
}

int qcb_flow_measure(qcb_flow fl, qcb_field src, int n_steps, int n_rk, double* tQE, double* plaq) {
    if (!fl || !src || !tQE || n_steps < 1 || n_rk < 0) return fail(QCB_EINVAL, "invalid argument");
    qcb_field_s* f = fl->fld;
    RET(qcb_field_copy(f, src));
    if ((size_t)n_steps > fl->meas_cap) {
        CK(cudaStreamSynchronize(f->stream));
        if (fl->d_meas) cudaFree(fl->d_meas);
        fl->d_meas = nullptr;
        fl->meas_cap = 0;
        CK(cudaMalloc(&fl->d_meas, (size_t)n_steps * 3 * sizeof(double)));
        fl->meas_cap = (size_t)n_steps;
    }
    if (!fl->d_count) CK(cudaMalloc(&fl->d_count, sizeof(int)));
    RET(ensure_alt(f));
    RET(ensure_partials(f, std::max((size_t)clover_blocks(f->g.Vh) * 18, (size_t)halves_blocks(f->g.Vh) * 3)));
#if QCB_FLOW_FUSED_MEAS
    // the clover halves of the measuring stage 1, allocated before any graph capture
    if (n_rk > 0 && !fl->halves) CK(cudaMalloc(&fl->halves, halves_bytes(f->fmt, f->g.Vh)));
#endif
    CK(cudaMemsetAsync(fl->d_count, 0, sizeof(int), f->stream));
    const bool graphs = graphs_ok(f) && n_rk > 0;
    for (int s = 0; s < n_steps; s++) {
        // measure (q, e and the plaquette sum), then n_rk RK3 steps unless this is the last time
        if (graphs && s != n_steps - 1)
            RET(flow_graph_run(fl, 2, n_rk));
        else
            RET(meas_block(fl, s != n_steps - 1 ? n_rk : 0));
    }
    std::vector<double> h((size_t)n_steps * 3);
    CK(cudaMemcpyAsync(h.data(), fl->d_meas, h.size() * sizeof(double), cudaMemcpyDeviceToHost, f->stream));
    CK(cudaStreamSynchronize(f->stream));
    double t = 0.0;
    for (int s = 0; s < n_steps; s++) {
        tQE[3 * s] = t;
        tQE[3 * s + 1] = h[3 * s];
        tQE[3 * s + 2] = h[3 * s + 1] / (double)f->g.V;
        if (plaq) plaq[s] = h[3 * s + 2] / (6.0 * (double)f->g.V);
        if (s != n_steps - 1)
            for (int k = 0; k < n_rk; k++) t += fl->eps;
    }
    return QCB_OK;
}

qcb_field qcb_flow_field(qcb_flow fl) { return fl ? fl->fld : nullptr; }

int qcb_flow_pass(qcb_flow fl, int pass) {
    if (!fl || pass < QCB_FLOW_FORCE0 || pass > QCB_FLOW_W3) return fail(QCB_EINVAL, "flow pass: invalid argument");
    qcb_field_s* f = fl->fld;
    if ((pass == QCB_FLOW_FORCE1 || pass == QCB_FLOW_W2 || pass == QCB_FLOW_REPLACE_F0 || pass == QCB_FLOW_W3) &&
        !fl->f1)
        CK(cudaMalloc(&fl->f1, alg_bytes(f->fmt, f->g.Vh)));
    const FmtOps& o = fmt_ops(f->fmt);
    const int rep = needs_reproject(f->prec, f->store);
    const double e = fl->eps;
    switch (pass) {
        case QCB_FLOW_FORCE0:
        case QCB_FLOW_FORCE1:
            return launch(f, QCB_K_FLOW, [&] {
                return o.flow_force(f->g, f->links, pass == QCB_FLOW_FORCE0 ? fl->z : fl->f1, f->stream);
            });
        case QCB_FLOW_W1:
            return launch(f, QCB_K_FLOW, [&] {
                return o.flow_update(f->g, f->links, fl->z, nullptr, 0.25 * e, 0.0, 0, 0, f->stream);
            });
        case QCB_FLOW_W2:
            return launch(f, QCB_K_FLOW, [&] {
                return o.flow_update(f->g, f->links, fl->z, fl->f1, (8.0 / 9.0) * e, (17.0 / 36.0) * e, 1, 0,
                                     f->stream);
            });
        case QCB_FLOW_REPLACE_F0:
            return launch(f, QCB_K_FLOW, [&] { return o.flow_replace(f->g, fl->z, fl->f1, f->stream); });
        default:
            return launch(f, QCB_K_FLOW, [&] {
                return o.flow_update(f->g, f->links, fl->z, fl->f1, 0.75 * e, e, 1, rep, f->stream);
            });
    }
}

// ------------------------------------------------------------------ instrumentation
int qcb_timing_enable(qcb_field f, int on) {
    if (!f) return fail(QCB_EINVAL, "null field");
    f->timing = on != 0;
    return QCB_OK;
}

int qcb_timing_read(qcb_field f, int kclass, long* launches, double* total_ms) {
    if (!f || kclass < 0 || kclass >= QCB_K_NCLASS) return fail(QCB_EINVAL, "invalid argument");
    CK(cudaStreamSynchronize(f->stream));
    for (auto& t : f->pending) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, t.a, t.b));
        f->t_count[t.kclass] += 1;
        f->t_ms[t.kclass] += ms;
        f->event_pool.push_back(t.a);
        f->event_pool.push_back(t.b);
    }
    f->pending.clear();
    if (launches) *launches = f->t_count[kclass];
    if (total_ms) *total_ms = f->t_ms[kclass];
    return QCB_OK;
}

int qcb_timing_reset(qcb_field f) {
    if (!f) return fail(QCB_EINVAL, "null field");
    long n;
    double ms;
    RET(qcb_timing_read(f, 0, &n, &ms));
    for (int k = 0; k < QCB_K_NCLASS; k++) {
        f->t_count[k] = 0;
        f->t_ms[k] = 0.0;
    }
    return QCB_OK;
}

// ------------------------------------------------------------------ diagnostics
int qcb_diag_staple(qcb_field f, int mu, double* out) {
    if (!f || !out || mu < 0 || mu > 3) return fail(QCB_EINVAL, "invalid argument");
    RET(staging_acquire(f));
    RET(launch(f, QCB_K_OTHER,
               [&] { return fmt_ops(f->fmt).staple_field(f->g, f->links, mu, f->staging, f->stream); }));
    CK(cudaMemcpyAsync(out, f->staging, (size_t)f->g.V * 9 * sizeof(double2), cudaMemcpyDeviceToHost, f->stream));
    RET(staging_release(f));
    CK(cudaStreamSynchronize(f->stream));
    return QCB_OK;
}

int qcb_diag_exp_su3(const double* Z, int n, double coeff, int prec, double* out) {
    if (!Z || !out || n < 0) return fail(QCB_EINVAL, "invalid argument");
    if (n == 0) return QCB_OK;
    double2 *dz = nullptr, *dout = nullptr;
    size_t bytes = (size_t)n * 9 * sizeof(double2);
    CK(cudaMalloc(&dz, bytes));
    cudaError_t e = cudaMalloc(&dout, bytes);
    if (e == cudaSuccess) e = cudaMemcpy(dz, Z, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_diag_exp<<<(n + 127) / 128, 128>>>(dz, n, coeff, prec == QCB_PREC_F32 ? 1 : 0, dout);
        g_launches.fetch_add(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, bytes, cudaMemcpyDeviceToHost);
    cudaFree(dz);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(QCB_ECUDA, "diag exp: %s", cudaGetErrorString(e));
    return QCB_OK;
}

int qcb_diag_fma_rate(int prec, double* flop_per_s) {
    if (!flop_per_s || (prec != QCB_PREC_F64 && prec != QCB_PREC_F32)) return fail(QCB_EINVAL, "invalid argument");
    void* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaMalloc(&out, sizeof(double)));
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    const int blocks = sm_count() * 8, threads = 256;
    const int iters = prec == QCB_PREC_F64 ? 1024 : 4096;
    float best = 0.f;
    for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
        e = cudaEventRecord(e0, 0);
        if (prec == QCB_PREC_F64)
            k_fma_rate<double><<<blocks, threads>>>(0.999999, 1e-7, iters, (double*)out);
        else
            k_fma_rate<float><<<blocks, threads>>>(0.999999f, 1e-7f, iters, (float*)out);
        g_launches.fetch_add(1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(e1, 0);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e == cudaSuccess && rep > 0 && (best == 0.f || ms < best)) best = ms;  // rep 0 warms up
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return fail(QCB_ECUDA, "fma rate: %s", cudaGetErrorString(e));
    const double fmas = (double)blocks * threads * iters * 4.0 * 8.0;
    *flop_per_s = 2.0 * fmas / (best * 1e-3);
    return QCB_OK;
}

int qcb_diag_philox(const uint32_t ctr[4], const uint32_t key[2], int n, uint32_t* out) {
    if (!ctr || !key || !out || n < 0) return fail(QCB_EINVAL, "invalid argument");
    if (n == 0) return QCB_OK;
    uint4* d = nullptr;
    CK(cudaMalloc(&d, (size_t)n * sizeof(uint4)));
    k_diag_philox<<<(n + 127) / 128, 128>>>(make_uint4(ctr[0], ctr[1], ctr[2], ctr[3]), make_uint2(key[0], key[1]), n,
                                           d);
    g_launches.fetch_add(1);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, d, (size_t)n * sizeof(uint4), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(QCB_ECUDA, "diag philox: %s", cudaGetErrorString(e));
    return QCB_OK;
}

}  // extern "C"
