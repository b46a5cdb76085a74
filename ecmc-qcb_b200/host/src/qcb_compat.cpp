// qcb_compat.cpp -- the reference's C++ hot-path signatures implemented over the libqcb C ABI.
#include <cstdio>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>

#include "flow/gradient_flow.h"
#include "gauge/GaugeField.h"
#include "heatbath/heatbath_mpi.h"
#include "io/ildg.h"
#include "mpi/Shift.h"
#include "observables/observables_mpi.h"

namespace fs = std::filesystem;

void qcb_check(int status, const char* what) {
    if (status != QCB_OK) throw std::runtime_error(std::string(what) + ": " + qcb_last_error());
}

namespace {
int lattice4(const GeometryCB& g, int L[4]) {
    for (int d = 0; d < 4; d++) L[d] = g.L_int;
    return 0;
}
}  // namespace

// ====================================================================== GaugeField
GaugeField::GaugeField(const GeometryCB& geo) : links(geo.V_ext * 4 * 9, Complex(0, 0)), geo_(geo) {
    int L[4];
    lattice4(geo, L);
    qcb_check(qcb_field_create(L, QCB_PREC_F64, QCB_STORE_18, &h_), "GaugeField");
    // identity everywhere, halo included (GaugeField.h:30-43)
    for (size_t s = 0; s < geo.V_ext; s++)
        for (int mu = 0; mu < 4; mu++)
            for (int i = 0; i < 3; i++) links[(s * 4 + mu) * 9 + 4 * i] = Complex(1, 0);
}

GaugeField::GaugeField(const GeometryCB& geo, qcb_field borrowed)
    : links(geo.V_ext * 4 * 9, Complex(0, 0)), geo_(geo), h_(borrowed), owns_(false), host_stale_(true) {}

GaugeField::GaugeField(const GaugeField& o) : links(), geo_(o.geo_) {
    int L[4];
    lattice4(geo_, L);
    qcb_check(qcb_field_create(L, QCB_PREC_F64, QCB_STORE_18, &h_), "GaugeField copy");
    qcb_check(qcb_field_copy(h_, o.device()), "GaugeField copy");
    links = o.links;
    host_stale_ = o.host_stale_;
}

GaugeField& GaugeField::operator=(const GaugeField& o) {
    if (this == &o) return *this;
    qcb_check(qcb_field_copy(h_, o.device()), "GaugeField assign");
    links = o.links;
    host_stale_ = o.host_stale_;
    dev_stale_ = false;
    return *this;
}

GaugeField::~GaugeField() {
    if (owns_ && h_) qcb_field_destroy(h_);
}

void GaugeField::upload_if_stale() const {
    if (!dev_stale_) return;
    const GeometryCB& g = geo_;
    const int L = g.L_int;
    std::vector<Complex> aos((size_t)g.V_int * 36);
    size_t k = 0;
    for (int t = 1; t <= L; t++)
        for (int z = 1; z <= L; z++)
            for (int y = 1; y <= L; y++)
                for (int x = 1; x <= L; x++) {
                    const Complex* src = &links[g.index(x, y, z, t) * 36];
                    for (int e = 0; e < 36; e++) aos[k++] = src[e];
                }
    qcb_check(qcb_field_upload_aos(h_, reinterpret_cast<const double*>(aos.data())), "upload");
    dev_stale_ = false;
}

void GaugeField::sync_host() const {
    if (!host_stale_) return;
    const GeometryCB& g = geo_;
    const int L = g.L_int;
    std::vector<Complex> aos((size_t)g.V_int * 36);
    qcb_check(qcb_field_download_aos(h_, reinterpret_cast<double*>(aos.data())), "download");
    auto& out = const_cast<std::vector<Complex>&>(links);
    // interior, then the halo as a periodic copy (the single-rank halo exchange)
    for (int t = 0; t < g.L_ext; t++)
        for (int z = 0; z < g.L_ext; z++)
            for (int y = 0; y < g.L_ext; y++)
                for (int x = 0; x < g.L_ext; x++) {
                    auto wrap = [L](int c) { return (c + L - 1) % L; };
                    const size_t src = (((size_t)wrap(t) * L + wrap(z)) * L + wrap(y)) * L + wrap(x);
                    Complex* dst = &out[g.index(x, y, z, t) * 36];
                    for (int e = 0; e < 36; e++) dst[e] = aos[src * 36 + e];
                }
    host_stale_ = false;
}

qcb_field GaugeField::device() const {
    upload_if_stale();
    return h_;
}
void GaugeField::mark_device_modified() { host_stale_ = true; }
void GaugeField::mark_host_modified() { dev_stale_ = true; }

SU3Map GaugeField::view_link(size_t site, int mu) {
    sync_host();
    dev_stale_ = true;  // the caller may write through the view
    return SU3Map{&links[(site * 4 + mu) * 9]};
}
SU3ConstMap GaugeField::view_link_const(size_t site, int mu) const {
    sync_host();
    return SU3ConstMap{&links[(site * 4 + mu) * 9]};
}

void GaugeField::hot_start(const GeometryCB&, std::mt19937_64& rng) {
    qcb_check(qcb_hot_start(h_, rng()), "hot_start");
    dev_stale_ = false;
    host_stale_ = true;
}
void GaugeField::cold_start(const GeometryCB&) {
    qcb_check(qcb_cold_start(h_), "cold_start");
    dev_stale_ = false;
    host_stale_ = true;
}

// projection_su3 (GaugeField.cpp:36-58) on one host link.
void GaugeField::projection_su3(size_t site, int mu) {
    SU3Map U = view_link(site, mu);
    Complex c0[3], c1[3];
    for (int i = 0; i < 3; i++) {
        c0[i] = U(i, 0);
        c1[i] = U(i, 1);
    }
    double n0 = std::sqrt(std::norm(c0[0]) + std::norm(c0[1]) + std::norm(c0[2]));
    for (auto& c : c0) c /= n0;
    Complex dot = std::conj(c0[0]) * c1[0] + std::conj(c0[1]) * c1[1] + std::conj(c0[2]) * c1[2];
    for (int i = 0; i < 3; i++) c1[i] -= c0[i] * dot;
    double n1 = std::sqrt(std::norm(c1[0]) + std::norm(c1[1]) + std::norm(c1[2]));
    for (auto& c : c1) c /= n1;
    for (int i = 0; i < 3; i++) {
        U(i, 0) = c0[i];
        U(i, 1) = c1[i];
    }
    U(0, 2) = std::conj(c0[1] * c1[2] - c0[2] * c1[1]);
    U(1, 2) = std::conj(c0[2] * c1[0] - c0[0] * c1[2]);
    U(2, 2) = std::conj(c0[0] * c1[1] - c0[1] * c1[0]);
}

void GaugeField::project_field_su3(const GeometryCB&) {
    qcb_check(qcb_reunitarize(device()), "project_field_su3");
    host_stale_ = true;
}

// compute_staple (GaugeField.cpp:74-97) of one link, on the host copy.
void GaugeField::compute_staple(const GeometryCB& geo, size_t site, int mu, SU3& staple) const {
    sync_host();
    staple.setZero();
    const size_t xmu = geo.get_neigh(site, mu, up);
    auto L = [&](size_t s, int m) { return SU3(SU3ConstMap{&links[(s * 4 + m) * 9]}); };
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        const size_t xnu = geo.get_neigh(site, nu, up);
        staple += L(xmu, nu) * (L(site, nu) * L(xnu, mu)).adjoint();
        const size_t xmunu = geo.get_neigh(xmu, nu, down);
        const size_t xmnu = geo.get_neigh(site, nu, down);
        staple += (L(xmnu, mu) * L(xmunu, nu)).adjoint() * L(xmnu, nu);
    }
}

// ====================================================================== heatbath
namespace mpi::heatbathcb {
void hit(GaugeField& field, const GeometryCB& geo, size_t site, int mu, double beta, SU3& A, std::mt19937_64& rng) {
    int c[4];
    geo.coords(site, c);
    int64_t lex = 0;
    for (int d = 3; d >= 0; d--) lex = lex * geo.L_int + (((c[d] - 1) % geo.L_int) + geo.L_int) % geo.L_int;
    const uint64_t key = rng();
    double a[18];
    qcb_check(qcb_hb_link(field.device(), lex, mu, beta, 1, key, 0u, a), "heatbath hit");
    for (int k = 0; k < 9; k++) A.m[k] = Complex(a[2 * k], a[2 * k + 1]);
    field.mark_device_modified();
}

void sweep(GaugeField& field, const GeometryCB&, double beta, int N_hits, std::vector<std::mt19937_64>& rng,
           site_parity update_parity) {
    if (!field.hb_seeded) {
        field.hb_seed = rng.empty() ? 0ull : rng[0]();
        field.hb_seeded = true;
    }
    qcb_field f = field.device();
    const int p = (update_parity == EV) ? 0 : 1;
    for (int mu = 0; mu < 4; mu++)
        qcb_check(qcb_hb_subsweep(f, beta, N_hits, field.hb_seed, field.hb_sweep, p, mu), "heatbath sweep");
    field.hb_sweep++;
    field.mark_device_modified();
}

std::vector<double> samples(GaugeField& field, const GeometryCB& geo, MpiTopology& topo, const HbParams& params,
                            std::vector<std::mt19937_64>& rng, parity active_parity) {
    std::vector<double> meas(params.N_samples);
    for (int m = 0; m < params.N_samples; m++)
        if (topo.p == active_parity)
            for (int s = 0; s < params.N_sweeps; s++) {
                sweep(field, geo, params.beta, params.N_hits, rng, EV);
                sweep(field, geo, params.beta, params.N_hits, rng, OD);
            }
    return meas;
}
}  // namespace mpi::heatbathcb

// ====================================================================== flow
namespace {
qcb_flow make_flow(const GaugeField& field, double eps) {
    qcb_flow fl = nullptr;
    qcb_check(qcb_flow_create(field.device(), eps, QCB_PREC_F64, QCB_STORE_18, &fl), "GradientFlow");
    return fl;
}
}  // namespace

GradientFlow::GradientFlow(double epsilon_, const GaugeField& field, const GeometryCB& geo)
    : epsilon(epsilon_),
      fl_(make_flow(field, epsilon_)),
      holder_(new GaugeField(geo, qcb_flow_field(fl_))),
      field_c(*holder_),
      geo_p(&geo) {}

GradientFlow::~GradientFlow() {
    holder_.reset();
    if (fl_) qcb_flow_destroy(fl_);
}

void GradientFlow::copy(const GaugeField& field) {
    qcb_check(qcb_flow_copy(fl_, field.device()), "GradientFlow::copy");
    field_c.mark_device_modified();
}

void GradientFlow::rk3_step(mpi::MpiTopology&) {
    field_c.device();  // host edits of field_c, if any
    qcb_check(qcb_flow_rk3(fl_, 1), "rk3_step");
    field_c.mark_device_modified();
}

// The reference's separate passes (gradient_flow.cpp:17-121), one C ABI pass each.
void GradientFlow::run_pass(int pass, const char* what) {
    field_c.device();
    qcb_check(qcb_flow_pass(fl_, pass), what);
    field_c.mark_device_modified();
}
void GradientFlow::compute_force(int i) { run_pass(i == 0 ? QCB_FLOW_FORCE0 : QCB_FLOW_FORCE1, "compute_force"); }
void GradientFlow::compute_w1() { run_pass(QCB_FLOW_W1, "compute_w1"); }
void GradientFlow::compute_w2() { run_pass(QCB_FLOW_W2, "compute_w2"); }
void GradientFlow::replace_force_0() { run_pass(QCB_FLOW_REPLACE_F0, "replace_force_0"); }
void GradientFlow::compute_w3() { run_pass(QCB_FLOW_W3, "compute_w3"); }

// ====================================================================== observables
namespace {
// Lexicographic index of the interior site a halo'd index names (halo sites wrap periodically).
int64_t interior_lex(const GeometryCB& geo, size_t site) {
    int c[4];
    geo.coords(site, c);
    int64_t lex = 0;
    for (int d = 3; d >= 0; d--) lex = lex * geo.L_int + (((c[d] - 1) % geo.L_int) + geo.L_int) % geo.L_int;
    return lex;
}
}  // namespace

namespace mpi::observables {
SU3 clover_site(const GaugeField& field, const GeometryCB& geo, size_t site, int mu, int nu) {
    double F[18];
    qcb_check(qcb_clover_site(field.device(), interior_lex(geo, site), mu, nu, F), "clover_site");
    SU3 r;
    for (int k = 0; k < 9; k++) r.m[k] = Complex(F[2 * k], F[2 * k + 1]);
    return r;
}

// observables_mpi.cpp:51-63: +1 / -1 for even / odd permutations of distinct indices, else 0.
int levi_civita(int mu, int nu, int rho, int sigma) {
    if (mu == nu || mu == rho || mu == sigma || nu == rho || nu == sigma || rho == sigma) return 0;
    const int inv = (mu > nu) + (mu > rho) + (mu > sigma) + (nu > rho) + (nu > sigma) + (rho > sigma);
    return (inv & 1) ? -1 : 1;
}

std::pair<double, double> local_q_e_clover(const GaugeField& field, const GeometryCB& geo, size_t site) {
    double q = 0.0, e = 0.0;
    qcb_check(qcb_local_qe(field.device(), interior_lex(geo, site), &q, &e), "local_q_e_clover");
    return {q, e};
}

double mean_plaquette_local(const GaugeField& field, const GeometryCB& geo) {
    double p = 0;
    qcb_check(qcb_plaquette(field.device(), &p), "plaquette");
    return p * 6.0 * (double)geo.V_int;
}
double mean_plaquette_global(GaugeField& field, const GeometryCB&, MpiTopology&) {
    double p = 0;
    qcb_check(qcb_plaquette(field.device(), &p), "plaquette");
    return p;
}
std::pair<double, double> topo_q_e_clover(const GaugeField& field, const GeometryCB& geo) {
    double q = 0, e = 0;
    qcb_check(qcb_clover_qe(field.device(), &q, &e), "clover");
    return {q, e * (double)geo.V_int};
}
std::pair<double, double> topo_q_e_clover_global(const GaugeField& field, const GeometryCB&, MpiTopology&) {
    double q = 0, e = 0;
    qcb_check(qcb_clover_qe(field.device(), &q, &e), "clover");
    return {q, e};
}

namespace {
std::string fmt(double v, int p) {
    std::stringstream ss;
    ss << std::fixed << std::setprecision(p) << v;
    return ss.str();
}
}  // namespace

// topo_charge_flowed (observables_mpi.cpp:159-186), including its progress lines on rank 0.
std::vector<double> topo_charge_flowed(GaugeField& field, const GeometryCB&, GradientFlow& gf, mpi::MpiTopology& topo,
                                       int N_steps_gf, int N_rk_steps) {
    std::vector<double> tQE(3 * (size_t)N_steps_gf);
    qcb_check(qcb_flow_measure(gf.handle(), field.device(), N_steps_gf, N_rk_steps, tQE.data(), nullptr),
              "topo_charge_flowed");
    gf.field_c.mark_device_modified();
    if (topo.rank == 0)
        for (int s = 0; s < N_steps_gf; s++) {
            const double t = tQE[3 * s], q = tQE[3 * s + 1], e = tQE[3 * s + 2];
            std::cout << "n = " << s << ", t = " << fmt(t, 2) << ", Q = " << fmt(q, 6)
                      << ", t²E = " << fmt(t * t * e, 6) << "\n";
        }
    return tQE;
}
}  // namespace mpi::observables

// ====================================================================== ILDG
namespace {
fs::path ildg_path(const std::string& filename, const std::string& dirpath) {
    return fs::path(dirpath) / filename / filename;
}
}  // namespace

void save_ildg_clime(const std::string& filename, const std::string& dirpath, const GaugeField& field,
                     const GeometryCB&, const mpi::MpiTopology& topo) {
    fs::path file = ildg_path(filename, dirpath);
    fs::create_directories(file.parent_path());
    qcb_check(qcb_ildg_write(field.device(), file.string().c_str()), "save_ildg_clime");
    if (topo.rank == 0) std::cout << "Configuration saved in " << file << "\n";
}

void read_ildg_clime(const std::string& filename, const std::string& dirpath, GaugeField& field, const GeometryCB&,
                     mpi::MpiTopology&) {
    fs::path file = ildg_path(filename, dirpath);
    qcb_check(qcb_ildg_read(field.device(), file.string().c_str()), "read_ildg_clime");
    field.mark_device_modified();
}

// ====================================================================== shift
namespace mpi::shift {
namespace {
int g_range = 0;
}
void set_shift_range(int range) { g_range = range; }

void shift_field(GaugeField& field, const GeometryCB&, HalosShift&, mpi::MpiTopology&, const int s[4]) {
    qcb_check(qcb_shift(field.device(), s), "shift_field");
    field.mark_device_modified();
}

void random_shift(GaugeField& field, const GeometryCB& geo, HalosShift& h, mpi::MpiTopology& topo,
                  std::mt19937_64& rng) {
    std::uniform_int_distribution<int> rand_l_shift(0, (g_range > 0 ? g_range : geo.L_int) - 1);
    int s[4];
    s[0] = rand_l_shift(rng);
    s[1] = rand_l_shift(rng);
    s[2] = rand_l_shift(rng);
    s[3] = rand_l_shift(rng);
    if (topo.rank == 0) std::cout << "Shift (" << s[0] << ", " << s[1] << ", " << s[2] << ", " << s[3] << ")\n";
    shift_field(field, geo, h, topo, s);
}
}  // namespace mpi::shift
