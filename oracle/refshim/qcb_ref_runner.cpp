// qcb_ref_runner.cpp -- C entry points over the reference's own hot-path code, compiled unchanged
// from the ECMC-QCB sources into oracle/_ref/libqcb_ref.so.  TEST INFRASTRUCTURE ONLY: tests and
// the golden-fixture script load it to pin the restated oracle and the CUDA path to what the
// reference itself computes.
//
// One lattice is the reference's one-rank layout: an (L+2)^4 GeometryCB box whose halo the
// reference's own exchange_halos_cascade fills periodically (the one-rank MPI stand-in sends each
// face to itself).  Fields cross this interface in the AoS order of the ILDG payload: interior
// sites x fastest, t slowest, 4 links per site, row-major 3x3 complex as (re, im) doubles,
//     U[(((lex*4 + mu)*9) + i*3 + j)*2 + {0, 1}],  lex = x + L*(y + L*(z + L*t)),
// which is the reference's own GaugeField::links order restricted to the interior.
//
// The heatbath entry points call the reference's mpi::heatbathcb::hit (src/heatbath/heatbath_mpi.cpp:10-33)
// link by link over one (parity, mu) set, with the std::mt19937_64 of each link replaced at compile
// time by the replay of that link's Philox stream (qcb_ref_rng.h): key = seed,
// counter = (call, lex*4 + mu, sweep, TAG_HB).  The set order and the stream keys are those of the
// CUDA path; the update arithmetic is the reference's.
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "flow/gradient_flow.h"
#include "gauge/GaugeField.h"
#include "geometry/GeometryCB.h"
#include "heatbath/heatbath_mpi.h"
#include "io/ildg.h"
#include "io/io.h"
#include "mpi/HalosExchange.h"
#include "mpi/HalosShift.h"
#include "mpi/MpiTopology.h"
#include "mpi/Shift.h"
#include "observables/observables_mpi.h"
#include "su3/utils.h"

// io::format_double is the one io.cpp routine the hot path calls (topo_charge_flowed prints its
// progress with it, src/observables/observables_mpi.cpp:175-177); io.cpp itself needs c-lime.
// Fixed notation with `precision` digits, as its declaration's callers use it.
std::string io::format_double(double val, int precision) {
    std::ostringstream os;
    os << std::fixed << std::setprecision(precision) << val;
    return os.str();
}

namespace {

struct RefLattice {
    int L;
    GeometryCB geo;
    GaugeField field;
    mpi::MpiTopology topo;
    HalosShift hs;
    explicit RefLattice(int L_) : L(L_), geo(L_), field(geo), topo(1), hs(geo) {}

    long volume() const { return (long)L * L * L * L; }
    void coords(long lex, int c[4]) const {
        c[0] = (int)(lex % L);
        c[1] = (int)((lex / L) % L);
        c[2] = (int)((lex / ((long)L * L)) % L);
        c[3] = (int)(lex / ((long)L * L * L));
    }
    size_t site(long lex) const {
        int c[4];
        coords(lex, c);
        return geo.index(c[0] + 1, c[1] + 1, c[2] + 1, c[3] + 1);
    }
    int parity(long lex) const {
        int c[4];
        coords(lex, c);
        return (c[0] + c[1] + c[2] + c[3]) & 1;
    }
    void halos() { mpi::exchange::exchange_halos_cascade(field, geo, topo); }
};

void put_matrix(double* out, const SU3& m) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            out[(i * 3 + j) * 2] = m(i, j).real();
            out[(i * 3 + j) * 2 + 1] = m(i, j).imag();
        }
}
SU3 get_matrix(const double* in) {
    SU3 m;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m(i, j) = Complex(in[(i * 3 + j) * 2], in[(i * 3 + j) * 2 + 1]);
    return m;
}

// Runs f with std::cout discarded (topo_charge_flowed prints one line per measurement).
template <class F>
void quiet(F f) {
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    f();
    std::cout.rdbuf(old);
}

// One link's hits through the reference's hit(); returns the staple A it computed last.
void hit_link(RefLattice& r, long lex, int mu, double beta, int n_hits, uint64_t seed, uint32_t sweep, SU3& A) {
    std::mt19937_64 rng(seed, (uint32_t)(lex * 4 + mu), sweep, qcb_ref::TAG_HB);  // the replay engine
    for (int h = 0; h < n_hits; h++) mpi::heatbathcb::hit(r.field, r.geo, r.site(lex), mu, beta, A, rng);
}

}  // namespace

extern "C" {

void* qref_create(int L) {
    if (L < 2 || L % 2) return nullptr;
    return new RefLattice(L);
}
void qref_destroy(void* h) { delete static_cast<RefLattice*>(h); }
void qref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// Interior links in, halos filled by the reference's cascade exchange.
void qref_set_aos(void* h, const double* U) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    for (long lex = 0; lex < r.volume(); lex++)
        for (int mu = 0; mu < 4; mu++)
            r.field.view_link(r.site(lex), mu) = get_matrix(U + ((size_t)lex * 4 + mu) * 18);
    r.halos();
}
void qref_get_aos(void* h, double* U) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    for (long lex = 0; lex < r.volume(); lex++)
        for (int mu = 0; mu < 4; mu++) put_matrix(U + ((size_t)lex * 4 + mu) * 18, r.field.view_link_const(r.site(lex), mu));
}

// GaugeField::compute_staple (src/gauge/GaugeField.cpp:74-97) at every site for one mu; out is V*18 doubles.
void qref_staple_field(void* h, int mu, double* out) {
    RefLattice& r = *static_cast<RefLattice*>(h);
#pragma omp parallel for schedule(static)
    for (long lex = 0; lex < r.volume(); lex++) {
        SU3 A;
        r.field.compute_staple(r.geo, r.site(lex), mu, A);
        put_matrix(out + (size_t)lex * 18, A);
    }
}

// mean_plaquette_global (src/observables/observables_mpi.cpp:11-48).
double qref_plaquette(void* h) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    return mpi::observables::mean_plaquette_global(r.field, r.geo, r.topo);
}

// topo_q_e_clover_global (src/observables/observables_mpi.cpp:115-156): Q and E = sum(e)/V.
void qref_clover_qe(void* h, double* Q, double* E) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    auto qe = mpi::observables::topo_q_e_clover_global(r.field, r.geo, r.topo);
    *Q = qe.first;
    *E = qe.second;
}

// local_q_e_clover (src/observables/observables_mpi.cpp:93-112) at every site.
void qref_clover_density(void* h, double* q, double* e) {
    RefLattice& r = *static_cast<RefLattice*>(h);
#pragma omp parallel for schedule(static)
    for (long lex = 0; lex < r.volume(); lex++) {
        auto qe = mpi::observables::local_q_e_clover(r.field, r.geo, r.site(lex));
        q[lex] = qe.first;
        e[lex] = qe.second;
    }
}

// clover_site (src/observables/observables_mpi.cpp:66-90) at one site.
void qref_clover_site(void* h, long lex, int mu, int nu, double* out18) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    put_matrix(out18, mpi::observables::clover_site(r.field, r.geo, r.site(lex), mu, nu));
}

// n GradientFlow::rk3_step calls (src/flow/gradient_flow.cpp:124-135) of size eps, in place.
void qref_flow_rk3(void* h, double eps, int n) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    GradientFlow gf(eps, r.field, r.geo);
    for (int k = 0; k < n; k++) gf.rk3_step(r.topo);
    r.field = gf.field_c;
}

// GradientFlow's member passes in the order given (0 compute_force(0), 1 compute_force(1),
// 2 compute_w1, 3 compute_w2, 4 replace_force_0, 5 compute_w3), with the halo exchange rk3_step
// makes after each update (src/flow/gradient_flow.cpp:124-135); the field becomes field_c.
void qref_flow_passes(void* h, double eps, const int* seq, int n) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    GradientFlow gf(eps, r.field, r.geo);
    for (int k = 0; k < n; k++) {
        switch (seq[k]) {
            case 0: gf.compute_force(0); break;
            case 1: gf.compute_force(1); break;
            case 2: gf.compute_w1(); break;
            case 3: gf.compute_w2(); break;
            case 4: gf.replace_force_0(); break;
            default: gf.compute_w3(); break;
        }
        if (seq[k] == 2 || seq[k] == 3 || seq[k] == 5) mpi::exchange::exchange_halos_cascade(gf.field_c, r.geo, r.topo);
    }
    r.field = gf.field_c;
}

// topo_charge_flowed (src/observables/observables_mpi.cpp:159-186); tQE holds 3*n_steps doubles.
// The field itself is left unflowed (the reference flows the GradientFlow's copy).
void qref_flow_measure(void* h, double eps, int n_steps, int n_rk, double* tQE) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    GradientFlow gf(eps, r.field, r.geo);
    std::vector<double> v;
    quiet([&] { v = mpi::observables::topo_charge_flowed(r.field, r.geo, gf, r.topo, n_steps, n_rk); });
    std::memcpy(tQE, v.data(), v.size() * sizeof(double));
}

// Every link (x, mu) with parity(x) == parity: n_hits calls of mpi::heatbathcb::hit on that
// link's Philox replay stream; then the halos are refreshed for the next set.
void qref_hb_subsweep(void* h, double beta, int n_hits, uint64_t seed, uint32_t sweep, int parity, int mu) {
    RefLattice& r = *static_cast<RefLattice*>(h);
#pragma omp parallel for schedule(static)
    for (long lex = 0; lex < r.volume(); lex++) {
        if (r.parity(lex) != parity) continue;
        SU3 A;
        hit_link(r, lex, mu, beta, n_hits, seed, sweep, A);
    }
    r.halos();
}

// The CUDA path's sweep order: (parity 0, mu 0..3) then (parity 1, mu 0..3).
void qref_hb_sweep(void* h, double beta, int n_hits, uint64_t seed, uint32_t sweep) {
    for (int p = 0; p < 2; p++)
        for (int mu = 0; mu < 4; mu++) qref_hb_subsweep(h, beta, n_hits, seed, sweep, p, mu);
}

// One link's hits; A_out receives the staple A the reference's hit() leaves in its argument.
void qref_hb_link(void* h, long lex, int mu, double beta, int n_hits, uint64_t seed, uint32_t sweep, double* A_out) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    SU3 A;
    hit_link(r, lex, mu, beta, n_hits, seed, sweep, A);
    if (A_out) put_matrix(A_out, A);
    r.halos();
}

// GaugeField::project_field_su3 (src/gauge/GaugeField.cpp:36-71).
void qref_projection(void* h) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    r.field.project_field_su3(r.geo);
    r.halos();
}

// mpi::shift::shift_field (src/mpi/Shift.cpp:109-160) with s[d] in [0, L]: U'(x) = U(x - s).
void qref_shift(void* h, const int s[4]) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    mpi::shift::shift_field(r.field, r.geo, r.hs, r.topo, s);
    r.halos();
}

// save_ildg_clime / read_ildg_clime (src/io/ildg.cpp:34-237): the file is dir/name/name, as the
// reference lays it out; the writer's run directory dir/name is created first (the reference's
// driver has made it by the time it saves).
int qref_ildg_write(void* h, const char* dir, const char* name) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    std::error_code ec;
    std::filesystem::create_directories(std::filesystem::path(dir) / name, ec);
    if (ec) return -1;
    quiet([&] { save_ildg_clime(name, dir, r.field, r.geo, r.topo); });
    return 0;
}
void qref_ildg_read(void* h, const char* dir, const char* name) {
    RefLattice& r = *static_cast<RefLattice*>(h);
    read_ildg_clime(name, dir, r.field, r.geo, r.topo);
}

// exp_su3_luscher (src/su3/utils.cpp:145-193) and proj_lie_su3 (:130-134) on one matrix.
void qref_exp_su3_luscher(const double* Z, double coeff, double* out) { put_matrix(out, exp_su3_luscher(get_matrix(Z), coeff)); }
void qref_proj_lie_su3(double* A) {
    SU3 m = get_matrix(A);
    proj_lie_su3(m);
    put_matrix(A, m);
}

}  // extern "C"
