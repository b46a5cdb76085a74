// qcb_batch.cu -- many independent heatbath chains advanced together.
//
// A batch holds n lattices of (possibly) different sizes and couplings in one device arena.
// Each (parity, mu) phase of a sweep is ONE persistent launch over the tile work list of all
// chains (k_hb_tiles); a whole sweep -- 8 phases plus the device-side sweep counter increment --
// is captured once as a CUDA graph and replayed.  Chain i draws from the Philox link streams
// keyed on its own seed, with the batch's sweep counter, so it receives exactly the numbers a
// single-lattice run (qcb_hb_sweep with the same seed and sweep index) would.
// The autotuner times the heatbath launch shapes (threads per block x resident blocks) on the
// live batch -- every shape computes the same links, so tuning sweeps are ordinary sweeps -- and
// optionally the 12-real storage on a converted copy.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

#include "qcb_internal.h"
#include "qcb_ops.h"

using namespace qcb;

struct qcb_batch_s {
    int n = 0;
    int prec = 64, store = 0, fmt = 0;
    std::vector<LatDesc> desc;          // host copy of the descriptors
    std::vector<double> beta;
    void* arena = nullptr;              // all link fields
    LatDesc* d_desc = nullptr;
    int* d_tile_lat = nullptr;
    int nb_total = 0;
    uint32_t* d_sweep = nullptr;        // device sweep counter (read by the graph's kernels)
    uint32_t sweep = 0;                 // host mirror
    double* partials = nullptr;
    double* d_out = nullptr;
    double* h_out = nullptr;
    double2* staging = nullptr;
    int64_t max_V = 0;
    int* d_err = nullptr;
    cudaStream_t stream = nullptr;
    int variant = 1;
    cudaGraphExec_t graph = nullptr;
    int graph_hits = -1, graph_variant = -1;
};

namespace {

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

__global__ void k_bump_sweep(uint32_t* s) { *s += 1u; }

WorkList batch_list(const qcb_batch_s* b) {
    WorkList w;
    w.lats = b->d_desc;
    w.tile_lat = b->n > 1 ? b->d_tile_lat : nullptr;
    if (b->n == 1) w.lats = b->d_desc;
    w.nb_total = b->nb_total;
    w.nlat = b->n;
    return w;
}

void drop_graph(qcb_batch_s* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_hits = b->graph_variant = -1;
}

// Lays out the arena for format fmt and fills descriptors + tile map (links not initialised).
int layout(qcb_batch_s* b, int fmt) {
    size_t total = 0;
    std::vector<size_t> off(b->n);
    for (int i = 0; i < b->n; i++) {
        off[i] = total;
        total += (link_bytes(fmt, b->desc[i].g.Vh) + 255) & ~(size_t)255;
    }
    void* arena = nullptr;
    cudaError_t e = cudaMalloc(&arena, total);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? QCB_ENOMEM : QCB_ECUDA, "batch arena (%zu bytes): %s", total,
                    cudaGetErrorString(e));
    if (b->arena) cudaFree(b->arena);
    b->arena = arena;
    b->fmt = fmt;
    b->store = (fmt & 1) ? QCB_STORE_12 : QCB_STORE_18;
    for (int i = 0; i < b->n; i++) b->desc[i].links = (char*)arena + off[i];
    CK(cudaMemcpy(b->d_desc, b->desc.data(), sizeof(LatDesc) * b->n, cudaMemcpyHostToDevice));
    drop_graph(b);
    return QCB_OK;
}

int run_phase_set(qcb_batch_s* b, int n_hits, int variant) {
    const WorkList w = batch_list(b);
    const int rep = needs_reproject(b->prec, b->store);
    for (int p = 0; p < 2; p++)
        for (int mu = 0; mu < 4; mu++) {
            cudaError_t e = fmt_ops(b->fmt).hb(w, variant, p, mu, n_hits, b->d_sweep, 0u, rep, b->d_err, b->stream);
            if (e != cudaSuccess) return fail(QCB_ECUDA, "batch heatbath launch: %s", cudaGetErrorString(e));
        }
    note_launches(8);
    return QCB_OK;
}

// One sweep executed eagerly (also warms the launchers' occupancy caches before a capture).
int sweep_eager(qcb_batch_s* b, int n_hits, int variant) {
    RET(run_phase_set(b, n_hits, variant));
    k_bump_sweep<<<1, 1, 0, b->stream>>>(b->d_sweep);
    CK(cudaGetLastError());
    note_launches(1);
    b->sweep++;
    return QCB_OK;
}

int capture(qcb_batch_s* b, int n_hits, int variant) {
    drop_graph(b);
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int r = run_phase_set(b, n_hits, variant);
    if (r == QCB_OK) {
        k_bump_sweep<<<1, 1, 0, b->stream>>>(b->d_sweep);
        if (cudaGetLastError() != cudaSuccess) r = fail(QCB_ECUDA, "capture: counter kernel");
    }
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (r != QCB_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(QCB_ECUDA, "end capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->graph = nullptr;
        return fail(QCB_ECUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    b->graph_hits = n_hits;
    b->graph_variant = variant;
    return QCB_OK;
}

// Copies every lattice of b into dst (same lattices, possibly another storage format).
int convert_into(qcb_batch_s* b, qcb_batch_s* dst) {
    if (!b->staging) CK(cudaMalloc(&b->staging, (size_t)b->max_V * 36 * sizeof(double2)));
    for (int i = 0; i < b->n; i++) {
        CK(fmt_ops(b->fmt).soa_to_aos(b->desc[i].g, b->desc[i].links, b->staging, 0, b->stream));
        CK(fmt_ops(dst->fmt).aos_to_soa(dst->desc[i].g, b->staging, dst->desc[i].links, 0, b->stream));
    }
    note_launches(2 * b->n);
    return QCB_OK;
}

int read_err(qcb_batch_s* b) {
    int h = 0;
    CK(cudaMemcpyAsync(&h, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    if (h) {
        CK(cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream));
        if (h & DERR_BULK_WAIT)
            return fail(QCB_ETIMEOUT, "heatbath: bulk copy of the block's links did not complete (links left unchanged)");
        if (h & DERR_KP_SCALE)
            return fail(QCB_ERANGE, "batch heatbath: zero or non-finite SU(2) projection of a staple");
        return fail(QCB_ERANGE, "batch heatbath: Kennedy-Pendleton attempt cap (2^20) reached");
    }
    return QCB_OK;
}

}  // namespace

extern "C" {

int qcb_batch_create(int n, const int* L, const double* beta, const uint64_t* seed, int prec, int store,
                     qcb_batch* out) {
    if (n < 1 || !L || !beta || !seed || !out) return fail(QCB_EINVAL, "batch: invalid argument");
    if (prec != QCB_PREC_F64 && prec != QCB_PREC_F32) return fail(QCB_EINVAL, "prec must be 64 or 32");
    if (store != QCB_STORE_18 && store != QCB_STORE_12) return fail(QCB_EINVAL, "store must be 0 or 1");
    for (int i = 0; i < n; i++) {
        if (!lattice_ok(L + 4 * i))
            return fail(QCB_EINVAL, "batch lattice %d: extents must be even, >= 2, volume <= 2^30", i);
        if (!(beta[i] > 0.0)) return fail(QCB_EINVAL, "batch lattice %d: beta must be > 0", i);
    }
    qcb_batch_s* b = new (std::nothrow) qcb_batch_s();
    if (!b) return fail(QCB_ENOMEM, "host allocation");
    b->n = n;
    b->prec = prec;
    b->desc.resize(n);
    b->beta.assign(beta, beta + n);
    std::vector<int> tile_lat;
    int nb = 0;
    for (int i = 0; i < n; i++) {
        LatDesc& d = b->desc[i];
        memset(&d, 0, sizeof(d));
        d.g = make_geom(L + 4 * i);
        d.c_alpha = -0.75 / beta[i];
        d.seed = seed[i];
        d.nb_begin = nb;
        d.nb = (int)((d.g.Vh + TILE - 1) / TILE);
        for (int k = 0; k < d.nb; k++) tile_lat.push_back(i);
        nb += d.nb;
        b->max_V = std::max<int64_t>(b->max_V, d.g.V);
    }
    b->nb_total = nb;
    int r = QCB_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_desc, sizeof(LatDesc) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_tile_lat, sizeof(int) * tile_lat.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_tile_lat, tile_lat.data(), sizeof(int) * tile_lat.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_sweep, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(b->d_sweep, 0, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->partials, sizeof(double) * 12 * (size_t)nb);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_out, sizeof(double) * 2 * n);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_out, sizeof(double) * 2 * n);
    if (e != cudaSuccess) {
        r = fail(e == cudaErrorMemoryAllocation ? QCB_ENOMEM : QCB_ECUDA, "batch allocation: %s",
                 cudaGetErrorString(e));
        qcb_batch_destroy(b);
        return r;
    }
    r = layout(b, fmt_of(prec, store));
    if (r != QCB_OK) {
        qcb_batch_destroy(b);
        return r;
    }
    *out = b;
    return qcb_batch_cold_start(b);
}

int qcb_batch_destroy(qcb_batch b) {
    if (!b) return QCB_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graph(b);
    if (b->arena) cudaFree(b->arena);
    if (b->d_desc) cudaFree(b->d_desc);
    if (b->d_tile_lat) cudaFree(b->d_tile_lat);
    if (b->d_sweep) cudaFree(b->d_sweep);
    if (b->d_err) cudaFree(b->d_err);
    if (b->partials) cudaFree(b->partials);
    if (b->d_out) cudaFree(b->d_out);
    if (b->h_out) cudaFreeHost(b->h_out);
    if (b->staging) cudaFree(b->staging);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return QCB_OK;
}

int qcb_batch_info(qcb_batch b, int* n, int* prec, int* store, int* variant, uint32_t* sweep) {
    if (!b) return fail(QCB_EINVAL, "null batch");
    if (n) *n = b->n;
    if (prec) *prec = b->prec;
    if (store) *store = b->store;
    if (variant) *variant = b->variant;
    if (sweep) *sweep = b->sweep;
    return QCB_OK;
}

void* qcb_batch_stream(qcb_batch b) { return b ? (void*)b->stream : nullptr; }

static int batch_start(qcb_batch b, int hot) {
    for (int i = 0; i < b->n; i++) {
        cudaError_t e = fmt_ops(b->fmt).start(b->desc[i].g, b->desc[i].links, hot, b->desc[i].seed, b->stream);
        if (e != cudaSuccess) return fail(QCB_ECUDA, "batch start: %s", cudaGetErrorString(e));
    }
    note_launches(b->n);
    return QCB_OK;
}

int qcb_batch_cold_start(qcb_batch b) {
    if (!b) return fail(QCB_EINVAL, "null batch");
    return batch_start(b, 0);
}

int qcb_batch_hot_start(qcb_batch b) {
    if (!b) return fail(QCB_EINVAL, "null batch");
    return batch_start(b, 1);
}

int qcb_batch_sweep(qcb_batch b, int n_hits, int n_sweeps) {
    if (!b || n_hits < 0 || n_sweeps < 0) return fail(QCB_EINVAL, "batch sweep: invalid argument");
    int done = 0;
    if (n_sweeps > 0 && (!b->graph || b->graph_hits != n_hits || b->graph_variant != b->variant)) {
        RET(sweep_eager(b, n_hits, b->variant));
        done = 1;
        if (done < n_sweeps) RET(capture(b, n_hits, b->variant));
    }
    for (; done < n_sweeps; done++) {
        CK(cudaGraphLaunch(b->graph, b->stream));
        note_launches(9);
        b->sweep++;
    }
    return QCB_OK;
}

int qcb_batch_sync(qcb_batch b) {
    if (!b) return fail(QCB_EINVAL, "null batch");
    return read_err(b);
}

int qcb_batch_plaquette(qcb_batch b, double* out) {
    if (!b || !out) return fail(QCB_EINVAL, "null argument");
    const WorkList w = batch_list(b);
    CK(fmt_ops(b->fmt).plaq_tiles(w, -1, b->partials, b->stream));
    k_lat_finalize<<<b->n, 256, 0, b->stream>>>(b->d_desc, LatDesc{}, b->partials, 2, 1, 1, b->d_out);
    CK(cudaGetLastError());
    note_launches(2);
    CK(cudaMemcpyAsync(b->h_out, b->d_out, sizeof(double) * b->n, cudaMemcpyDeviceToHost, b->stream));
    RET(read_err(b));
    memcpy(out, b->h_out, sizeof(double) * b->n);
    return QCB_OK;
}

int qcb_batch_upload_aos(qcb_batch b, int i, const double* links) {
    if (!b || !links || i < 0 || i >= b->n) return fail(QCB_EINVAL, "batch upload: invalid argument");
    if (!b->staging) CK(cudaMalloc(&b->staging, (size_t)b->max_V * 36 * sizeof(double2)));
    const Geom& g = b->desc[i].g;
    CK(cudaMemcpyAsync(b->staging, links, (size_t)g.V * 36 * sizeof(double2), cudaMemcpyHostToDevice, b->stream));
    CK(fmt_ops(b->fmt).aos_to_soa(g, b->staging, b->desc[i].links, 0, b->stream));
    note_launches(1);
    CK(cudaStreamSynchronize(b->stream));
    return QCB_OK;
}

int qcb_batch_download_aos(qcb_batch b, int i, double* links) {
    if (!b || !links || i < 0 || i >= b->n) return fail(QCB_EINVAL, "batch download: invalid argument");
    if (!b->staging) CK(cudaMalloc(&b->staging, (size_t)b->max_V * 36 * sizeof(double2)));
    const Geom& g = b->desc[i].g;
    CK(fmt_ops(b->fmt).soa_to_aos(g, b->desc[i].links, b->staging, 0, b->stream));
    note_launches(1);
    CK(cudaMemcpyAsync(links, b->staging, (size_t)g.V * 36 * sizeof(double2), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return QCB_OK;
}

int qcb_batch_set_variant(qcb_batch b, int variant) {
    if (!b || variant < 0 || variant >= kHbVariants) return fail(QCB_EINVAL, "batch: variant out of range");
    b->variant = variant;
    return QCB_OK;
}

// Autotuner: times n_trial sweeps of every heatbath launch shape on the live batch (identical
// results for every shape) and keeps the fastest; with allow_store_change, also times the
// other link storage (18 <-> 12 reals) on a converted copy and switches if it is faster.
// ms_out (may be NULL) receives kHbVariants + 1 times per sweep: the shapes in the current
// storage, then the best shape in the other storage (0 if not tried).
int qcb_batch_tune(qcb_batch b, int n_hits, int n_trial, int allow_store_change, int* variant_out, double* ms_out) {
    if (!b || n_hits < 0 || n_trial < 1) return fail(QCB_EINVAL, "batch tune: invalid argument");
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double best = 1e300, times[kHbVariants + 1] = {0};
    int best_v = b->variant;
    for (int v = 0; v < kHbVariants; v++) {
        RET(sweep_eager(b, n_hits, v));  // warm-up (and occupancy query outside the timing)
        cudaEventRecord(e0, b->stream);
        for (int k = 0; k < n_trial; k++) RET(sweep_eager(b, n_hits, v));
        cudaEventRecord(e1, b->stream);
        CK(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        times[v] = ms / n_trial;
        if (times[v] < best) {
            best = times[v];
            best_v = v;
        }
    }
    b->variant = best_v;
    if (allow_store_change) {
        // time the other storage on a converted copy of the whole batch
        const int other = b->fmt ^ 1;
        qcb_batch_s tmp;
        tmp.n = b->n;
        tmp.prec = b->prec;
        tmp.desc = b->desc;
        tmp.beta = b->beta;
        tmp.nb_total = b->nb_total;
        tmp.stream = b->stream;
        tmp.d_sweep = b->d_sweep;
        tmp.d_err = b->d_err;
        tmp.d_tile_lat = b->d_tile_lat;
        int r = QCB_OK;
        cudaError_t ce = cudaMalloc(&tmp.d_desc, sizeof(LatDesc) * b->n);
        if (ce != cudaSuccess) r = fail(QCB_ENOMEM, "tune: descriptors");
        if (r == QCB_OK) r = layout(&tmp, other);
        if (r == QCB_OK) r = convert_into(b, &tmp);
        const uint32_t saved = b->sweep;
        if (r == QCB_OK) r = sweep_eager(&tmp, n_hits, best_v);
        if (r == QCB_OK) {
            cudaEventRecord(e0, b->stream);
            for (int k = 0; k < n_trial && r == QCB_OK; k++) r = sweep_eager(&tmp, n_hits, best_v);
            cudaEventRecord(e1, b->stream);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            times[kHbVariants] = ms / n_trial;
        }
        // the trial sweeps on the copy advanced the shared device counter; restore it
        cudaMemcpyAsync(b->d_sweep, &saved, sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream);
        cudaStreamSynchronize(b->stream);
        if (r == QCB_OK && times[kHbVariants] < best) {
            // switch storage: convert the batch's (untouched) current links again and adopt them
            r = convert_into(b, &tmp);
            if (r == QCB_OK) {
                cudaStreamSynchronize(b->stream);
                if (b->arena) cudaFree(b->arena);
                b->arena = tmp.arena;
                tmp.arena = nullptr;
                b->fmt = tmp.fmt;
                b->store = tmp.store;
                b->desc = tmp.desc;
                cudaMemcpy(b->d_desc, b->desc.data(), sizeof(LatDesc) * b->n, cudaMemcpyHostToDevice);
                drop_graph(b);
                best = times[kHbVariants];
            }
        }
        if (tmp.arena) cudaFree(tmp.arena);
        if (tmp.d_desc) cudaFree(tmp.d_desc);
        tmp.stream = nullptr;
        tmp.d_tile_lat = nullptr;
        tmp.d_sweep = nullptr;
        tmp.d_err = nullptr;
        RET(r);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (variant_out) *variant_out = b->variant;
    if (ms_out)
        for (int k = 0; k <= kHbVariants; k++) ms_out[k] = times[k];
    return read_err(b);
}

}  // extern "C"
