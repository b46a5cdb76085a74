// qcb_internal.h -- host-side internals shared by the C ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>

#include <string>
#include <vector>

#include "../../include/qcb.h"
#include "qcb_field.cuh"

namespace qcb {

// Storage format of a field: index into {D18, D12, F18, F12}.
enum Fmt : int { FMT_D18 = 0, FMT_D12 = 1, FMT_F18 = 2, FMT_F12 = 3 };
inline int fmt_of(int prec, int store) { return (prec == QCB_PREC_F32 ? 2 : 0) + (store == QCB_STORE_12 ? 1 : 0); }
inline int fmt_ne(int fmt) { return (fmt & 1) ? 6 : 9; }
inline size_t fmt_cbytes(int fmt) { return (fmt & 2) ? sizeof(float2) : sizeof(double2); }
// Device bytes of a link field / su(3) accumulator in the tiled layout (32-site tiles).
inline size_t tiled_sites(int64_t Vh) { return (size_t)((Vh + 31) / 32) * 32; }
inline size_t link_bytes(int fmt, int64_t Vh) { return (size_t)8 * fmt_ne(fmt) * tiled_sites(Vh) * fmt_cbytes(fmt); }
inline size_t alg_bytes(int fmt, int64_t Vh) { return (size_t)8 * 4 * tiled_sites(Vh) * fmt_cbytes(fmt); }
// Device bytes of the clover halves a measuring stage 1 writes: per site 6 planes x 2 halves x 9
// reals and 6 plaquette traces (HalfClovers in qcb_kernels.cuh), in the link precision.
constexpr int kHalfCloverReals = 6 * 2 * 9 + 6;
inline size_t halves_bytes(int fmt, int64_t Vh) { return (size_t)kHalfCloverReals * 2 * Vh * (fmt_cbytes(fmt) / 2); }
// Blocks of the per-site sum of the clover halves (one thread per site, 128 a block).
inline unsigned halves_blocks(int64_t Vh) { return (unsigned)((2 * Vh + 127) / 128); }

// Lattice extents every entry point accepts: even, >= 2, at most 2^30 sites.  The running volume
// is checked after each factor (and every factor is at most 2^30), so no product overflows.
inline bool lattice_ok(const int* L, int64_t* V_out = nullptr) {
    int64_t V = 1;
    for (int d = 0; d < 4; d++) {
        if (L[d] < 2 || (L[d] & 1) || L[d] > (1 << 30)) return false;
        V *= L[d];
        if (V > ((int64_t)1 << 30)) return false;
    }
    if (V_out) *V_out = V;
    return true;
}

// Site blocks (grid y) of the single-lattice clover pass: one block of 128 threads per 128 half-sites,
// up to the grid's y limit (a grid-stride loop covers the rest).  Every clover pass of a lattice uses
// this count, so its partial sums and their order are the same on every path.
inline unsigned clover_blocks(int64_t Vh) {
    const int64_t nb = (Vh + 127) / 128;
    return (unsigned)(nb < 65535 ? nb : 65535);
}

int fail(int code, const char* fmt, ...);
// Adds n to the process-wide kernel launch counter reported by qcb_launch_count().
void note_launches(int n);

struct TimedLaunch {
    int kclass;
    cudaEvent_t a, b;
};

}  // namespace qcb

// FP64 reprojection after every link update: always for FP32 links, and for 12-real storage in
// either precision, whose rebuilt third row conj(r0 x r1) makes an SU(3) matrix only from
// orthonormal rows; without it the norm errors of the stored rows grow under the updates (an FP64
// 12-real heatbath chain diverged after ~180 sweeps).
inline int needs_reproject(int prec, int store) { return (prec == QCB_PREC_F32 || store == QCB_STORE_12) ? 1 : 0; }

struct qcb_field_s {
    int L[4];
    qcb::Geom g;
    int prec, store, fmt;
    int device;
    void* links = nullptr;  // current link buffer
    void* alt = nullptr;    // second link buffer (shift target), lazily allocated
    double2* staging = nullptr;  // device AoS staging buffer, lazily allocated
    cudaStream_t copy_stream = nullptr;  // host -> staging copies of qcb_field_prefetch_aos
    cudaEvent_t ev_copied = nullptr;     // end of the latest prefetch copy
    cudaEvent_t ev_staging = nullptr;    // end of the staging buffer's latest use on `stream`
    bool staging_used = false;           // ev_staging has been recorded
    bool prefetch_pending = false;       // a prefetched configuration waits in staging for its commit
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double* partials = nullptr;
    size_t partials_cap = 0;  // doubles
    double* d_res = nullptr;  // device results (8 doubles)
    double* h_res = nullptr;  // pinned host results (8 doubles)
    int* d_err = nullptr;     // device error flags
    bool timing = false;
    std::vector<qcb::TimedLaunch> pending;
    std::vector<cudaEvent_t> event_pool;
    long t_count[QCB_K_NCLASS] = {0};
    double t_ms[QCB_K_NCLASS] = {0};
};

// A captured sequence of a flow's launches, replayed with cudaGraphLaunch.  The launches bake in
// device pointers, so a graph is reused only for the same buffers: the link buffer it starts from,
// the reduction partials and the measurement buffer.
struct FlowGraph {
    cudaGraphExec_t exec = nullptr;
    int kind = 0;  // 1: two RK3 steps; 2: one measurement + n_rk RK3 steps
    int n_rk = 0;
    int kernels = 0;  // kernels one replay launches
    const void* links = nullptr;
    const void* partials = nullptr;
    const void* meas = nullptr;
    uint64_t last_use = 0;
};

struct qcb_flow_s {
    qcb_field_s* fld = nullptr;  // flowed field (owned); fld->links holds W
    void* wtmp = nullptr;         // ping-pong partner of fld->links
    void* z = nullptr;            // su(3) accumulator, 8 reals per link (force_0 of the separate passes)
    void* f1 = nullptr;           // force_1 of the separate passes, allocated at their first use
    double eps = 0.02;
    double* d_meas = nullptr;     // measurement rows (t-independent: q, e, plaquette sums) of qcb_flow_measure
    size_t meas_cap = 0;          // rows
    int* d_count = nullptr;       // device row counter of the measurement graphs
    void* halves = nullptr;       // clover halves of a measuring stage 1 (halves_bytes), at first use
    FlowGraph graphs[4];
    uint64_t graph_clock = 0;
};

namespace qcb {
// Raw AoS transfers used by the ILDG reader / writer.
int field_upload_host(qcb_field_s* f, const double* host, int bswap);
int field_download_host(qcb_field_s* f, double* host, int bswap);
}  // namespace qcb
