/*
 * qcb_oracle.h -- CPU restatement of the ECMC-QCB gauge-field hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle the CUDA product in
 * ecmc-qcb_b200/ is checked against: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  Nothing in
 * the product links or calls it.
 *
 * Parity status: PINNED to the reference's own code.  The reference ships no tests, golden
 * vectors or sample configuration, and its CMake build fetches Eigen and c-lime over the network.
 * Its hot-path sources are instead compiled unchanged (oracle/Makefile `ref`) against
 * project-written stand-ins for the Eigen API subset they use, a one-rank MPI and a Philox replay
 * engine in place of std::mt19937_64, into oracle/_ref/libqcb_ref.so.  tests/test_ref_pin.py
 * holds this restatement to that library (staples, plaquette, clover Q/E, RK3 steps, flow
 * measurement, heatbath sets and chained sweeps, shift, projection) and to fixtures it wrote
 * (tests/golden/ref_4444.npz), within 1e-12; they agree bit for bit except for the last bit of
 * the order-dependent global sums.  Analytic known answers (cold start, abelian plaquette, exp of
 * diagonal su(3) elements, Philox known-answer vectors) are checked in tests/test_oracle.py.
 *
 * Layout used by every function ("AoS"): a periodic L0*L1*L2*L3 lattice with
 * no halo, sites in lexicographic order with x fastest and t slowest, 4
 * links per site (mu = x,y,z,t), each a row-major 3x3 complex matrix stored
 * as (re, im) doubles:
 *     U[ (((site*4 + mu)*9) + i*3 + j)*2 + {0: re, 1: im} ]
 * This is the ILDG binary payload order (reference src/io/ildg.cpp:87-106)
 * in native byte order.
 *
 * Random numbers: the reference draws from std::mt19937_64 per OpenMP thread
 * (src/bin/gauge_hb_cb.cpp:31-36).  Both this oracle and the GPU replace it
 * with a counter-based Philox4x32-10 stream per link, keyed on the seed and
 * countered on (draw, link, sweep, tag), so results do not depend on thread
 * count or launch shape.
 */
#ifndef QCB_ORACLE_H
#define QCB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Philox4x32-10 (Salmon et al., SC'11); ctr[4], key[2] -> out[4]. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Number of OpenMP threads the oracle uses (0 = library default). */
void orc_set_threads(int n);
int orc_get_threads(void);

/* ---- single-matrix pieces (src/su3/utils.cpp) ---- */
void orc_exp_su3_luscher(const double* Z, double coeff, double* out);   /* utils.cpp:145-193 */
void orc_proj_lie_su3(double* A);                                       /* utils.cpp:130-134 */
void orc_projection_su3(double* U);                                     /* GaugeField.cpp:36-58 */

/* ---- field starts (GaugeField.cpp:10-33) ---- */
void orc_cold_start(double* U, const int L[4]);
void orc_hot_start(double* U, const int L[4], uint64_t seed);

/* ---- stencils ---- */
/* staple A(x,mu) of every site for one direction; out is V*9 complex.   GaugeField.cpp:74-97 */
void orc_staple_field(const double* U, const int L[4], int mu, double* out);
/* sum over sites of Re Tr(plaquettes)/3 divided by 6V.   observables_mpi.cpp:11-48 */
double orc_plaquette(const double* U, const int L[4]);
/* total clover charge Q and energy density E = sum(e)/V.   observables_mpi.cpp:66-156 */
void orc_clover_qe(const double* U, const int L[4], double* Q, double* E);
/* per-site clover charge density q(x) and energy e(x), each V doubles. */
void orc_clover_qe_density(const double* U, const int L[4], double* q, double* e);

/* ---- Wilson flow (gradient_flow.cpp:17-135) ---- */
/* n RK3 steps of size eps applied in place, with the reference's pass structure
   (force, update and replace_force_0 as separate sweeps over the lattice). */
void orc_flow_rk3(double* U, const int L[4], double eps, int n);
/* topo_charge_flowed (observables_mpi.cpp:159-186): flows a copy of U; tQE is 3*n_steps. */
void orc_flow_measure(const double* U, const int L[4], double eps, int n_steps, int n_rk,
                      double* tQE);

/* ---- heatbath (heatbath.cpp:8-44, heatbath_mpi.cpp:10-57) ---- */
/* update every link (x,mu) with parity(x)==parity, n_hits CM hits each. */
void orc_hb_subsweep(double* U, const int L[4], double beta, int n_hits, uint64_t seed,
                     uint32_t sweep, int parity, int mu);
/* full sweep: (parity 0, mu 0..3) then (parity 1, mu 0..3). */
void orc_hb_sweep(double* U, const int L[4], double beta, int n_hits, uint64_t seed,
                  uint32_t sweep);
/* Same updates as orc_hb_sweep, with the reference's cost structure: the
   staple is recomputed for every hit (heatbath_mpi.cpp:12) and the full
   3x3 products W = U*A and R*U are formed.  Used as the timed CPU baseline. */
void orc_hb_sweep_refcost(double* U, const int L[4], double beta, int n_hits, uint64_t seed,
                          uint32_t sweep);

void orc_hb_subsweep_refcost(double* U, const int L[4], double beta, int n_hits, uint64_t seed,
                             uint32_t sweep, int parity, int mu);

/* ---- global shift (Shift.cpp:109-186) ---- */
void orc_shift(double* U, const int L[4], const int s[4]);             /* U'(x) = U(x - s) */
void orc_random_shift_draw(uint64_t seed, uint64_t idx, const int L[4], int max_shift,
                           int s_out[4]);

/* ---- unitarity (GaugeField.cpp:61-71; src/bin/test.cpp:47-93) ---- */
void orc_reunitarize(double* U, const int L[4]);
void orc_unitarity(const double* U, const int L[4], double* max_err, double* mean_err);

#ifdef __cplusplus
}
#endif

#endif
