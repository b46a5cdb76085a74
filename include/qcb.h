/*
 * qcb.h -- C ABI of the B200 gauge-field hot path (libqcb.so).
 *
 * Plain pointers, sizes and opaque handles; no CUDA or C++ types cross it.  Every
 * function returns 0 (QCB_OK) or a negative status, never throws, and records a
 * message readable with qcb_last_error() (per host thread).  Work is ordered on the
 * handle's CUDA stream; calls that return results to host memory synchronise it.
 *
 * Host link buffers use the "AoS" order of the reference's GaugeField interior and of
 * the ILDG payload (src/gauge/GaugeField.h:27,49-56; src/io/ildg.cpp:87-106): sites
 * lexicographic with x fastest and t slowest, then mu = x,y,z,t, then the row-major
 * 3x3 complex matrix as (re, im) doubles -- V*4*9*2 doubles.
 *
 * Replaced reference interfaces are cited as path:line inside the reference tree.
 */
#ifndef QCB_H
#define QCB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define QCB_OK 0
#define QCB_EINVAL -1   /* invalid argument (sizes, parity, handle) */
#define QCB_ENOMEM -2   /* device allocation failed or over the configured budget */
#define QCB_EIO -3      /* file could not be opened / read / written */
#define QCB_EFORMAT -4  /* LIME/ILDG structure or size mismatch */
#define QCB_ECUDA -5    /* CUDA runtime error */
#define QCB_ETIMEOUT -6 /* a bounded device or host wait ran out */
#define QCB_ERANGE -7   /* a device-side cap was hit (e.g. heatbath attempt cap) */

/* ---- storage formats ---- */
#define QCB_PREC_F64 64
#define QCB_PREC_F32 32
#define QCB_STORE_18 0 /* full 3x3 complex matrix (18 reals) */
#define QCB_STORE_12 1 /* first two rows (12 reals), third rebuilt in registers; links in this
                          * storage (and FP32 links) are reprojected to SU(3) in FP64 after every
                          * heatbath update and every RK3 step */

typedef struct qcb_field_s* qcb_field;
typedef struct qcb_flow_s* qcb_flow;
typedef struct qcb_batch_s* qcb_batch;
typedef struct qcb_server_s* qcb_server;

/* Message of the last failing call on this host thread ("" if none). */
const char* qcb_last_error(void);
/* Library build string (arch, version). */
const char* qcb_version(void);
/* Number of kernels this library has launched in this process. */
uint64_t qcb_launch_count(void);

/* ------------------------------------------------------------------ fields */
/* Replaces GaugeField(const GeometryCB&) (src/gauge/GaugeField.h:30-43) and
 * GeometryCB(int L) (src/geometry/GeometryCB.cpp:5-9): one periodic L[0]xL[1]xL[2]xL[3]
 * lattice resident on the current CUDA device, every link set to the identity.  All
 * extents must be even and >= 2.  prec: QCB_PREC_F64 / QCB_PREC_F32; store: QCB_STORE_*. */
int qcb_field_create(const int L[4], int prec, int store, qcb_field* out);
int qcb_field_destroy(qcb_field f);
int qcb_field_info(qcb_field f, int L[4], int* prec, int* store, size_t* device_bytes);
/* The CUDA stream (cudaStream_t) the handle's work is ordered on, and a way to set it. */
void* qcb_field_stream(qcb_field f);
int qcb_field_set_stream(qcb_field f, void* cuda_stream);
int qcb_field_sync(qcb_field f);

/* Host <-> device in AoS order (see top).  Replaces direct access to GaugeField::links
 * (src/gauge/GaugeField.h:27).  `links` may be pageable or pinned host memory. */
int qcb_field_upload_aos(qcb_field f, const double* links);
int qcb_field_download_aos(qcb_field f, double* links);
/* Pipelined upload.  qcb_field_prefetch_aos starts copying an AoS configuration into the field's
 * staging buffer on a copy stream of its own and returns; the copy overlaps whatever the field's
 * stream is running (the links are not touched).  qcb_field_commit_prefetch then enqueues, on the
 * field's stream, the conversion of the copied configuration into the links, after the copy ends.
 * From pinned memory the copy is asynchronous, and the host buffer must stay unchanged until a
 * call after the commit has synchronised the field (qcb_field_sync, or any call that returns a
 * result); from pageable memory the copy is staged before the prefetch returns.  While a
 * prefetched configuration waits for its commit, the calls that need the staging buffer
 * (qcb_field_upload_aos / download_aos, a second prefetch, ILDG I/O, a copy between formats)
 * return QCB_EINVAL. */
int qcb_field_prefetch_aos(qcb_field f, const double* links);
int qcb_field_commit_prefetch(qcb_field f);
/* Same, from / to device memory (AoS doubles already on the field's device). */
int qcb_field_upload_aos_device(qcb_field f, const double* d_links);
int qcb_field_download_aos_device(qcb_field f, double* d_links);
/* dst <- src (any precision / storage combination; same lattice). */
int qcb_field_copy(qcb_field dst, qcb_field src);

/* cold_start (src/gauge/GaugeField.cpp:23-33). */
int qcb_cold_start(qcb_field f);
/* hot_start (src/gauge/GaugeField.cpp:10-20): Haar-random SU(3) per link from a Philox
 * stream keyed on seed (the reference's Householder-QR generator needs Eigen). */
int qcb_hot_start(qcb_field f, uint64_t seed);
/* project_field_su3 (src/gauge/GaugeField.cpp:61-71), column Gram-Schmidt in FP64. */
int qcb_reunitarize(qcb_field f);
/* max and mean over links of ||U U^dag - 1||_F (src/bin/test.cpp:47-93). */
int qcb_unitarity(qcb_field f, double* max_err, double* mean_err);

/* ------------------------------------------------------------------ global shift */
/* shift_field (src/mpi/Shift.cpp:109-160) on one periodic lattice: U'(x) = U(x - s). */
int qcb_shift(qcb_field f, const int s[4]);
/* random_shift (src/mpi/Shift.cpp:163-186): draws s_d uniform in [0, n-1] with
 * n = max_shift (or L[d] when max_shift <= 0) from a Philox stream keyed on (seed, idx),
 * applies it and returns it in s_out (may be NULL). */
int qcb_random_shift(qcb_field f, uint64_t seed, uint64_t idx, int max_shift, int s_out[4]);

/* ------------------------------------------------------------------ heatbath */
/* mpi::heatbathcb::sweep restricted to one (parity, mu) set (src/heatbath/heatbath_mpi.cpp:36-57,
 * hit :10-33, heatbath.cpp:8-44).  Every link (x, mu) with parity(x) == parity receives
 * n_hits Cabibbo-Marinari hits over the subgroups (0,1),(1,2),(0,2), with uniforms from a
 * Philox stream keyed on seed and countered on (draw, link, sweep). */
int qcb_hb_subsweep(qcb_field f, double beta, int n_hits, uint64_t seed, uint32_t sweep, int parity, int mu);
/* mpi::heatbathcb::hit (src/heatbath/heatbath_mpi.cpp:10-33, declared heatbath_mpi.h:14) on one
 * link: site is the lexicographic index x + L0*(y + L1*(z + L2*t)) of the periodic lattice.  The
 * link receives n_hits Cabibbo-Marinari hits with exactly the arithmetic and the Philox stream
 * (seed, sweep) that qcb_hb_subsweep gives it; A_out (may be NULL) receives the link's staple,
 * 9 complex as 18 doubles, row-major -- what hit() leaves in its SU3& A argument.  Synchronises
 * the field's stream. */
int qcb_hb_link(qcb_field f, int64_t site, int mu, double beta, int n_hits, uint64_t seed, uint32_t sweep,
                double* A_out);
/* Full sweep: (parity 0, mu 0..3) then (parity 1, mu 0..3).  Replaces the pair
 * sweep(EV); sweep(OD) of mpi::heatbathcb::samples (heatbath_mpi.cpp:60-75).  FP32 fields and
 * 12-real fields are reprojected to SU(3) in FP64 after each link update. */
int qcb_hb_sweep(qcb_field f, double beta, int n_hits, uint64_t seed, uint32_t sweep);

/* ------------------------------------------------------------------ observables */
/* mean_plaquette_global (src/observables/observables_mpi.cpp:39-48). */
int qcb_plaquette(qcb_field f, double* plaq);
/* topo_q_e_clover_global (src/observables/observables_mpi.cpp:136-156): Q and E = sum(e)/V. */
int qcb_clover_qe(qcb_field f, double* Q, double* E);
/* clover_site (src/observables/observables_mpi.cpp:66-90): the clover field strength
 * F_mu_nu = (C - C^dag)/8 at one site (lexicographic index), 9 complex as 18 doubles, row-major. */
int qcb_clover_site(qcb_field f, int64_t site, int mu, int nu, double* F_out);
/* local_q_e_clover (src/observables/observables_mpi.cpp:93-112) at one site: the topological charge
 * density q (with its 1/(4 pi^2)) and the energy density e. */
int qcb_local_qe(qcb_field f, int64_t site, double* q, double* e);

/* ------------------------------------------------------------------ Wilson flow */
/* GradientFlow(double eps, const GaugeField&, const GeometryCB&) (src/flow/gradient_flow.h:11-27,
 * gradient_flow.cpp:12-13): a flow state owning its flowed field and RK3 buffers, of the
 * given precision / storage (independent of src's), initialised as a copy of src. */
int qcb_flow_create(qcb_field src, double eps, int prec, int store, qcb_flow* out);
int qcb_flow_destroy(qcb_flow fl);
/* GradientFlow::copy (gradient_flow.cpp:138). */
int qcb_flow_copy(qcb_flow fl, qcb_field src);
/* n x GradientFlow::rk3_step (gradient_flow.cpp:124-135); fused stages, ping-pong buffers. */
int qcb_flow_rk3(qcb_flow fl, int n);
/* topo_charge_flowed (src/observables/observables_mpi.cpp:159-186): copy src, then n_steps
 * times { measure (Q, E) ; if not last: n_rk RK3 steps }; tQE receives 3*n_steps doubles
 * (t, Q, E).  If plaq is non-NULL it receives n_steps plaquettes measured beside Q, E.  With
 * n_rk > 0 every measurement is taken from a measuring RK3 stage 1 (the clover from the force's
 * staple differences): that of the step that follows it, for the last one a stage 1 whose output
 * is left unused; with n_rk = 0, from a clover pass.  The first call with n_rk > 0 allocates the
 * flow state's buffer for it (114 reals a site in the flow's precision). */
int qcb_flow_measure(qcb_flow fl, qcb_field src, int n_steps, int n_rk, double* tQE, double* plaq);
/* The flowed field (GradientFlow::field_c); owned by the flow state. */
qcb_field qcb_flow_field(qcb_flow fl);
/* GradientFlow's separate member passes (src/flow/gradient_flow.cpp:17-121, declared
 * gradient_flow.h:21-25) on the flowed field, for callers that drive them one by one (qcb_flow_rk3
 * runs the fused stages): force_0 and force_1 are su(3) fields of the flow state.
 *   QCB_FLOW_FORCE0 / FORCE1   compute_force(0 / 1): F = proj_lie_su3(-U A)
 *   QCB_FLOW_W1                compute_w1: U <- exp(eps/4 F0) U
 *   QCB_FLOW_W2                compute_w2: U <- exp(8/9 eps F1 - 17/36 eps F0) U
 *   QCB_FLOW_REPLACE_F0        replace_force_0: F0 <- 8/9 F1 - 17/36 F0
 *   QCB_FLOW_W3                compute_w3: U <- exp(3/4 eps F1 - eps F0) U
 * The reference's rk3_step is FORCE0, W1, FORCE1, W2, REPLACE_F0, FORCE1, W3 (its halo exchanges
 * are implicit on one GPU).  FP32 and 12-real links are reprojected after QCB_FLOW_W3, as after a
 * fused RK3 step. */
#define QCB_FLOW_FORCE0 0
#define QCB_FLOW_FORCE1 1
#define QCB_FLOW_W1 2
#define QCB_FLOW_W2 3
#define QCB_FLOW_REPLACE_F0 4
#define QCB_FLOW_W3 5
int qcb_flow_pass(qcb_flow fl, int pass);

/* ------------------------------------------------------------------ ILDG */
/* save_ildg_clime (src/io/ildg.cpp:34-136): LIME records "ildg-format" (MB=1, ME=1) and
 * "ildg-binary-data" (MB=0, ME=1), big-endian FP64, site order t,z,y,x, mu = x,y,z,t. */
int qcb_ildg_write(qcb_field f, const char* path);
/* qcb_ildg_write with flags.  QCB_ILDG_SCIDAC_CHECKSUM appends a "scidac-checksum" record
 * (MB=0, ME=1; the binary record then has ME=0) holding the SciDAC suma/sumb of the payload. */
#define QCB_ILDG_SCIDAC_CHECKSUM 1
int qcb_ildg_write_ex(qcb_field f, const char* path, int flags);
/* read_ildg_clime (src/io/ildg.cpp:138-237): finds "ildg-binary-data", checks its size
 * against the lattice, reads 64- or 32-bit payloads (precision from the "ildg-format"
 * record when present).  A "scidac-checksum" record, when the file has one, is checked
 * against the payload (QCB_EFORMAT on a mismatch). */
int qcb_ildg_read(qcb_field f, const char* path);
/* Reads the lattice extents and precision of an ILDG file ("ildg-format" record). */
int qcb_ildg_probe(const char* path, int L[4], int* precision);
/* SciDAC (USQCD QIO) checksums of a payload of n_sites records of site_bytes bytes in rank
 * order, bytes as stored: c_r = CRC-32 (zlib) of record r, suma = XOR rotl(c_r, r mod 29),
 * sumb = XOR rotl(c_r, r mod 31).  Host-only; needs no device. */
int qcb_scidac_checksum(const void* payload, uint64_t n_sites, uint64_t site_bytes, uint32_t* suma, uint32_t* sumb);

/* ------------------------------------------------------------------ instrumentation */
/* Kernel classes timed by CUDA events recorded on the handle's stream around each launch. */
#define QCB_K_HB 0
#define QCB_K_FLOW 1
#define QCB_K_PLAQ 2
#define QCB_K_CLOVER 3
#define QCB_K_OTHER 4
#define QCB_K_NCLASS 5
int qcb_timing_enable(qcb_field f, int on);
/* Synchronises and returns (launches, total ms) for one kernel class since the last reset. */
int qcb_timing_read(qcb_field f, int kclass, long* launches, double* total_ms);
int qcb_timing_reset(qcb_field f);

/* ------------------------------------------------------------------ checked build */
/* libqcb_checked.so is this library built with QCB_CHECKED: every (mu, parity, h) that a link
 * or su(3)-algebra access is formed from is validated on the device first; a bad one is counted,
 * the first kept, and the access redirected inside the field, so a kernel with an indexing error
 * reports it instead of faulting.  qcb_debug_oob synchronises the device and returns (and clears)
 * the count and the first bad access, packed as kind << 62 | (mu & 63) << 56 | (parity & 255) << 48
 * | (h mod 2^48) with kind 0 = link, 1 = algebra; *checked is 0 (and the count 0) in the normal
 * build. */
int qcb_debug_oob(int* checked, uint64_t* count, uint64_t* first);
/* Loads link (mu, parity, h) in a one-thread kernel.  The normal build rejects an index outside
 * the field on the host (QCB_EINVAL); the checked build passes it to the device check. */
int qcb_debug_probe_link(qcb_field f, int mu, int parity, int64_t h);

/* ------------------------------------------------------------------ diagnostics */
/* Staple A(x, mu) of every site (src/gauge/GaugeField.cpp:74-97) into host AoS (V*9 complex). */
int qcb_diag_staple(qcb_field f, int mu, double* out);
/* exp_su3_luscher (src/su3/utils.cpp:145-193) of n matrices (n*9 complex) on the device. */
int qcb_diag_exp_su3(const double* Z, int n, double coeff, int prec, double* out);
/* Measured fused multiply-add throughput of the current device in FLOP/s (2 per FMA), FP64 or FP32
 * (prec = QCB_PREC_F64 / QCB_PREC_F32): independent FMA chains on every SM, best of three timed
 * launches after a warm-up, on the legacy default stream.  The denominator of the flow kernels'
 * pipe fractions.  No counterpart in the reference. */
int qcb_diag_fma_rate(int prec, double* flop_per_s);
/* n Philox4x32-10 blocks on the device: ctr word 0 = ctr[0] + i. */
int qcb_diag_philox(const uint32_t ctr[4], const uint32_t key[2], int n, uint32_t* out);

/* ------------------------------------------------------------------ batched chains */
/* Many independent heatbath chains (the reference runs one chain per MPI job: src/bin/gauge_hb_cb.cpp
 * generate_hb_cb :20-247) advanced together on one GPU.  n lattices, extents L[4i..4i+3] (even,
 * >= 2), couplings beta[i], stream seeds seed[i], one storage format; all links start cold.
 * Chain i draws exactly what qcb_hb_sweep(field_i, beta[i], n_hits, seed[i], sweep) would for the
 * batch's sweep counter (0, 1, 2, ...). */
int qcb_batch_create(int n, const int* L, const double* beta, const uint64_t* seed, int prec, int store,
                     qcb_batch* out);
int qcb_batch_destroy(qcb_batch b);
int qcb_batch_info(qcb_batch b, int* n, int* prec, int* store, int* variant, uint32_t* sweep);
void* qcb_batch_stream(qcb_batch b);
/* hot_start / cold_start of every chain (chain i as qcb_hot_start(field, seed[i])). */
int qcb_batch_hot_start(qcb_batch b);
int qcb_batch_cold_start(qcb_batch b);
/* n_sweeps full sweeps of every chain.  Each (parity, mu) phase of all chains is one persistent
 * launch over a tile work list; one sweep (8 phases + the device sweep counter) is captured as a
 * CUDA graph at the first call with a given n_hits / launch shape and replayed. */
int qcb_batch_sweep(qcb_batch b, int n_hits, int n_sweeps);
/* Waits for queued work and reports a device-side heatbath error (QCB_ERANGE). */
int qcb_batch_sync(qcb_batch b);
/* Mean plaquette of every chain (out: n doubles). */
int qcb_batch_plaquette(qcb_batch b, double* out);
int qcb_batch_upload_aos(qcb_batch b, int i, const double* links);
int qcb_batch_download_aos(qcb_batch b, int i, double* links);
/* Launch shape of the heatbath phases (0: 64 threads, 1: 128, 2: 256 per block). */
int qcb_batch_set_variant(qcb_batch b, int variant);
/* Autotuner: times n_trial sweeps of every launch shape on the live batch (all shapes compute the
 * same links, so these are ordinary sweeps of the chains) and keeps the fastest; with
 * allow_store_change it also times the other link storage (18 <-> 12 reals) on a converted copy
 * and adopts it if faster.  ms_out (may be NULL): 4 times per sweep (3 shapes, other storage). */
int qcb_batch_tune(qcb_batch b, int n_hits, int n_trial, int allow_store_change, int* variant_out, double* ms_out);

/* ------------------------------------------------------------------ flow-measurement server */
/* Continuous-batching service for topo_charge_flowed (src/observables/observables_mpi.cpp:159-186):
 * requests of any lattice size are queued, admitted in order as the HBM budget allows, and every
 * scheduler tick measures (Q, E) of all resident requests and advances them by n_rk RK3 steps in
 * shared persistent launches.  Runs its own scheduler thread on the current device.
 * max_active <= 0: no limit besides the budget.  Every request takes its measurements from
 * measuring RK3 stage 1 launches, as qcb_flow_measure does; a request below 2^17 half-sites holds
 * 114 reals a site for them within its memory, and for the larger ones, which run alone, the server
 * keeps scratch outside the budget: 114 reals a site of the largest, in the server's precision. */
int qcb_serve_create(size_t hbm_budget_bytes, int prec, int store, int n_rk, int max_active, qcb_server* out);
int qcb_serve_destroy(qcb_server s);
/* Server options.  QCB_SERVE_GRAPHS (default 1): while the resident set of small requests is
 * unchanged from one tick to the next, their shared launches of a tick (the measuring stage 1 with
 * the halves' sums and the per-request finalize, then the rest of the n_rk RK3 steps) are replayed
 * from CUDA graphs captured for that set; 0 launches them one by one.  Results are the same either
 * way. */
#define QCB_SERVE_GRAPHS 1
int qcb_serve_set_option(qcb_server s, int option, int value);
/* Seconds on the server's clock (the clock of the times returned by qcb_serve_poll). */
double qcb_serve_now(qcb_server s);
/* Queues one request (thread-safe): host AoS FP64 links of an L[0..3] lattice, flow step eps,
 * n_steps measurements at t = 0, n_rk*eps, ... (n_steps - 1 flow blocks).  The links are copied. */
int qcb_serve_submit(qcb_server s, uint64_t id, const int L[4], const double* links, double eps, int n_steps);
/* Pops one completed request: returns 1 and fills id, tQE (3 * min(max_steps, n_steps) doubles:
 * t, Q, E), n_steps and times[3] = (submitted, admitted, completed); returns 0 if none is ready. */
int qcb_serve_poll(qcb_server s, uint64_t* id, double* tQE, int max_steps, int* n_steps, double* times);
/* Waits at most timeout_s seconds for every submitted request to complete (QCB_ETIMEOUT otherwise). */
int qcb_serve_wait(qcb_server s, double timeout_s);
/* out[8]: submitted, completed, scheduler rounds (a tick of the big requests and 1-8 ticks of the
 * small ones), peak resident, peak bytes, bytes in use, busy s, queued. */
int qcb_serve_stats(qcb_server s, double* out);

/* ------------------------------------------------------------------ allocation-free entry */
/* No counterpart in the reference (its plaquette, observables_mpi.cpp:39-48, runs on host
 * memory).  For callers that cannot let a library allocate device memory -- code inside a
 * framework that owns all device memory through its own pool, hosts that forbid allocation
 * after start-up, loops that must not hit the allocator's implicit synchronisation -- this
 * computes the mean plaquette of links the caller already holds in device memory and writes
 * it to device memory the caller provides (d_plaq[0]), enqueued on `stream` (NULL = legacy
 * default stream), without calling cudaMalloc, cudaFree or any allocating routine.
 * d_links: FP64 links in the parity-split layout of a QCB_PREC_F64 / QCB_STORE_18 field:
 *   complex element (row r, col c) of link (x, mu) at d_links[2*(((mu*2 + p)*9 + 3r + c)*V/2 + lex(x)/2)]
 *   (+1 for the imaginary part), lex(x) = x0 + L0*(x1 + L1*(x2 + L2*x3)), p = (x0+x1+x2+x3) mod 2.
 * d_links must be 16-byte aligned (its (re, im) pairs are read as 16-byte words) and d_plaq 8-byte
 * aligned; other pointers are refused with QCB_EINVAL.
 * Limits: even extents >= 2, volume <= 2^30 sites.  Scratch: a fixed static device array of
 * 2*148*8 doubles (18.5 KiB) that every GPU loading the library holds until exit; all calls
 * share it and it keeps the last call's contents, so calls that overlap on the GPU race.  The
 * first call on a device looks the array's address up (cudaGetSymbolAddress) with that device
 * current; make it before any stream capture on that device.  The address is kept for the life of
 * the process, so resetting the device (cudaDeviceReset) between calls is not supported. */
int qcb_plaquette_noalloc(const int L[4], const double* d_links, double* d_plaq, void* stream);

#ifdef __cplusplus
}
#endif

#endif
