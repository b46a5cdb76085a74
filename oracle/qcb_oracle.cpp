// qcb_oracle.cpp -- CPU restatement of the ECMC-QCB hot path (test infrastructure only).
//
// Every routine below follows one reference routine operation for operation;
// the reference file:line is given beside it (paths relative to the
// yacobozdalkiran/ECMC-QCB source tree).  The only deliberate departures are
//   * periodic neighbour arithmetic on one lattice instead of the halo'd
//     (L+2)^4 box + MPI halo exchange (src/geometry/GeometryCB.cpp:10-31,
//     src/mpi/HalosExchange.cpp:4-72): same neighbours, no frozen links;
//   * (parity, mu) update sets instead of the reference's racy "all mu of one
//     parity in one OpenMP loop" (src/heatbath/heatbath_mpi.cpp:36-57);
//   * a counter-based Philox4x32-10 stream per link instead of
//     std::mt19937_64 per thread (src/bin/gauge_hb_cb.cpp:31-36), and our own
//     Haar SU(3) generator for hot starts (the reference's Householder-QR
//     generator, src/su3/utils.cpp:13-30, needs Eigen's QR).
// Parity: pinned to the reference's own hot-path sources, compiled unchanged into
// oracle/_ref/libqcb_ref.so (tests/test_ref_pin.py), and to analytic known answers
// (tests/test_oracle.py).
#include "qcb_oracle.h"

#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// ---------------------------------------------------------------- complex / SU(3)
struct Cx {
    double re, im;
};
inline Cx cx(double r, double i) { return Cx{r, i}; }
inline Cx operator+(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
inline Cx operator-(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
inline Cx operator*(Cx a, Cx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline Cx operator*(double s, Cx a) { return cx(s * a.re, s * a.im); }
inline Cx conj(Cx a) { return cx(a.re, -a.im); }

struct M3 {
    Cx m[9];
    Cx& operator()(int i, int j) { return m[i * 3 + j]; }
    const Cx& operator()(int i, int j) const { return m[i * 3 + j]; }
};

inline M3 zero3() {
    M3 r;
    for (auto& e : r.m) e = cx(0, 0);
    return r;
}
inline M3 ident3() {
    M3 r = zero3();
    r(0, 0) = r(1, 1) = r(2, 2) = cx(1, 0);
    return r;
}
// Fixed-size 3x3 product, coefficient (i,j) = sum_k a(i,k) b(k,j) with k in index order.
inline M3 mul(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r(i, j) = (a(i, 0) * b(0, j) + a(i, 1) * b(1, j)) + a(i, 2) * b(2, j);
    return r;
}
inline M3 adj(const M3& a) {
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r(i, j) = conj(a(j, i));
    return r;
}
inline M3 add(const M3& a, const M3& b) {
    M3 r;
    for (int k = 0; k < 9; k++) r.m[k] = a.m[k] + b.m[k];
    return r;
}
inline M3 sub(const M3& a, const M3& b) {
    M3 r;
    for (int k = 0; k < 9; k++) r.m[k] = a.m[k] - b.m[k];
    return r;
}
inline M3 scale(double s, const M3& a) {
    M3 r;
    for (int k = 0; k < 9; k++) r.m[k] = s * a.m[k];
    return r;
}
inline Cx trace(const M3& a) { return (a(0, 0) + a(1, 1)) + a(2, 2); }
// 3x3 determinant by cofactor expansion along the first row.
inline Cx det3(const M3& m) {
    return (m(0, 0) * (m(1, 1) * m(2, 2) - m(1, 2) * m(2, 1)) -
            m(0, 1) * (m(1, 0) * m(2, 2) - m(1, 2) * m(2, 0))) +
           m(0, 2) * (m(1, 0) * m(2, 1) - m(1, 1) * m(2, 0));
}

// ---------------------------------------------------------------- lattice
struct Lat {
    int L[4];
    long V;
    explicit Lat(const int* l) {
        for (int d = 0; d < 4; d++) L[d] = l[d];
        V = (long)L[0] * L[1] * L[2] * L[3];
    }
    void coords(long s, int c[4]) const {
        c[0] = (int)(s % L[0]);
        s /= L[0];
        c[1] = (int)(s % L[1]);
        s /= L[1];
        c[2] = (int)(s % L[2]);
        c[3] = (int)(s / L[2]);
    }
    long index(const int c[4]) const { return ((long)(c[3] * L[2] + c[2]) * L[1] + c[1]) * L[0] + c[0]; }
    // periodic neighbour: GeometryCB::get_neigh (GeometryCB.cpp:10-31) on a periodic lattice.
    long neigh(long s, int mu, int dir) const {
        int c[4];
        coords(s, c);
        c[mu] += dir;
        if (c[mu] < 0) c[mu] += L[mu];
        if (c[mu] >= L[mu]) c[mu] -= L[mu];
        return index(c);
    }
    int parity(long s) const {
        int c[4];
        coords(s, c);
        return (c[0] + c[1] + c[2] + c[3]) & 1;
    }
};

inline M3 load(const double* U, long s, int mu) {
    M3 r;
    std::memcpy(r.m, U + (s * 4 + mu) * 18, sizeof(r.m));
    return r;
}
inline void store(double* U, long s, int mu, const M3& a) { std::memcpy(U + (s * 4 + mu) * 18, a.m, sizeof(a.m)); }

// ---------------------------------------------------------------- Philox4x32-10
inline void philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
        uint64_t p0 = (uint64_t)M0 * c0, p1 = (uint64_t)M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

// Stream tags (word 3 of the counter) -- identical constants in the CUDA product.
const uint32_t TAG_HB = 0x48420001u;     // heatbath link stream
const uint32_t TAG_HOT = 0x484F5401u;    // hot start link stream
const uint32_t TAG_SHIFT = 0x53480001u;  // random global shift

// 64 random bits -> double in [0,1) with 53 significant bits.
inline double u53(uint32_t hi, uint32_t lo) {
    uint64_t v = ((uint64_t)hi << 32) | lo;
    return (double)(v >> 11) * 0x1.0p-53;
}

// Per-link uniform stream: each Philox call yields two doubles, consumed in order.
struct LinkStream {
    uint32_t key[2];
    uint32_t ctr[4];
    double spare;
    bool has_spare;
    LinkStream(uint64_t seed, uint32_t link, uint32_t sweep, uint32_t tag) {
        key[0] = (uint32_t)seed;
        key[1] = (uint32_t)(seed >> 32);
        ctr[0] = 0;
        ctr[1] = link;
        ctr[2] = sweep;
        ctr[3] = tag;
        has_spare = false;
        spare = 0;
    }
    double next() {
        if (has_spare) {
            has_spare = false;
            return spare;
        }
        uint32_t o[4];
        philox(ctr, key, o);
        ctr[0]++;
        spare = u53(o[2], o[3]);
        has_spare = true;
        return u53(o[0], o[1]);
    }
};

// ---------------------------------------------------------------- su3 utils
// proj_lie_su3 -- src/su3/utils.cpp:130-134
inline void proj_lie_su3(M3& A) {
    M3 B = scale(0.5, sub(A, adj(A)));
    Cx tr = trace(B);
    Cx tr3 = cx(tr.re / 3.0, tr.im / 3.0);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            // B - tr3 * Identity
            Cx t = (i == j) ? tr3 : tr3 * cx(0.0, 0.0);
            A(i, j) = B(i, j) - t;
        }
}

// exp_su3_luscher -- src/su3/utils.cpp:145-193 (Cayley-Hamilton + Horner, N = 18)
inline M3 exp_su3_luscher(const M3& Z, double coeff) {
    M3 X = scale(coeff, Z);
    M3 X2 = mul(X, X);
    double t = -0.5 * trace(X2).re;
    Cx dt = det3(X);
    double d = (cx(0.0, 1.0) * dt).re;
    const int N = 18;
    double c[N + 1];
    c[0] = 1.0;
    for (int n = 1; n <= N; ++n) c[n] = c[n - 1] / (double)n;
    Cx q0 = cx(c[N], 0.0), q1 = cx(0.0, 0.0), q2 = cx(0.0, 0.0);
    for (int n = N - 1; n >= 0; --n) {
        Cx id = cx(0.0 * d, 1.0 * d);  // 1.0i * d
        Cx q0n = cx(c[n], 0.0) - id * q2;
        Cx q1n = q0 - t * q2;
        Cx q2n = q1;
        q0 = q0n;
        q1 = q1n;
        q2 = q2n;
    }
    M3 R;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            Cx idij = (i == j) ? cx(1.0, 0.0) : cx(0.0, 0.0);
            R(i, j) = (q0 * idij + q1 * X(i, j)) + q2 * X2(i, j);
        }
    return R;
}

// projection_su3 -- src/gauge/GaugeField.cpp:36-58 (column Gram-Schmidt)
inline void projection_su3(M3& U) {
    Cx c0[3], c1[3], c2[3];
    for (int i = 0; i < 3; i++) {
        c0[i] = U(i, 0);
        c1[i] = U(i, 1);
    }
    double n0 = std::sqrt((c0[0].re * c0[0].re + c0[0].im * c0[0].im) +
                          (c0[1].re * c0[1].re + c0[1].im * c0[1].im) +
                          (c0[2].re * c0[2].re + c0[2].im * c0[2].im));
    for (int i = 0; i < 3; i++) c0[i] = cx(c0[i].re / n0, c0[i].im / n0);
    Cx dot = (conj(c0[0]) * c1[0] + conj(c0[1]) * c1[1]) + conj(c0[2]) * c1[2];
    for (int i = 0; i < 3; i++) c1[i] = c1[i] - c0[i] * dot;
    double n1 = std::sqrt((c1[0].re * c1[0].re + c1[0].im * c1[0].im) +
                          (c1[1].re * c1[1].re + c1[1].im * c1[1].im) +
                          (c1[2].re * c1[2].re + c1[2].im * c1[2].im));
    for (int i = 0; i < 3; i++) c1[i] = cx(c1[i].re / n1, c1[i].im / n1);
    c2[0] = conj(c0[1] * c1[2] - c0[2] * c1[1]);
    c2[1] = conj(c0[2] * c1[0] - c0[0] * c1[2]);
    c2[2] = conj(c0[0] * c1[1] - c0[1] * c1[0]);
    for (int i = 0; i < 3; i++) {
        U(i, 0) = c0[i];
        U(i, 1) = c1[i];
        U(i, 2) = c2[i];
    }
}

// ---------------------------------------------------------------- SU(2) quaternions
struct Q4 {
    double a[4];
};
// su2_to_quaternion -- src/su3/utils.cpp:47-50, on the 2x2 block (w00 w01; w10 w11)
inline Q4 su2_to_quaternion(Cx w00, Cx w01, Cx w10, Cx w11) {
    return Q4{{(w00 + w11).re / 2.0, (w01 + w10).im / 2.0, (w01 - w10).re / 2.0, (w00 - w11).im / 2.0}};
}
// mult -- src/su3/utils.cpp:53-60
inline Q4 qmult(const Q4& q, const Q4& p) {
    return Q4{{q.a[0] * p.a[0] - q.a[1] * p.a[1] - q.a[2] * p.a[2] - q.a[3] * p.a[3],
               q.a[0] * p.a[1] + q.a[1] * p.a[0] + q.a[2] * p.a[3] - q.a[3] * p.a[2],
               q.a[0] * p.a[2] - q.a[1] * p.a[3] + q.a[2] * p.a[0] + q.a[3] * p.a[1],
               q.a[0] * p.a[3] + q.a[1] * p.a[2] - q.a[2] * p.a[1] + q.a[3] * p.a[0]}};
}
// adj -- src/su3/utils.cpp:63
inline Q4 qadj(const Q4& q) { return Q4{{q.a[0], -q.a[1], -q.a[2], -q.a[3]}}; }
// su2_quaternion_to_su3 -- src/su3/utils.cpp:33-44
inline M3 su2_quaternion_to_su3(const Q4& q, int i, int j) {
    M3 X = zero3();
    int k = 3 - i - j;
    X(k, k) = cx(1.0, 0.0);
    X(i, i) = cx(q.a[0], q.a[3]);
    X(j, j) = cx(q.a[0], -q.a[3]);
    X(i, j) = cx(q.a[2], q.a[1]);
    X(j, i) = cx(-q.a[2], q.a[1]);
    return X;
}

// generate_su2_kp -- src/heatbath/heatbath.cpp:8-36 (Kennedy-Pendleton)
inline Q4 generate_su2_kp(double beta, double k, LinkStream& rng) {
    double alpha = beta * k * 2.0 / 3.0;
    double a0;
    while (true) {
        double delta = rng.next();
        double r1 = rng.next();
        double r2 = rng.next();
        double r3 = rng.next();
        double c = std::cos(2 * M_PI * r2);
        double lambda_sq = -0.5 / alpha * (std::log(r1) + (c * c) * std::log(r3));
        if (delta * delta <= 1.0 - lambda_sq) {
            a0 = 1.0 - 2.0 * lambda_sq;
            break;
        }
    }
    double r_spatial = std::sqrt(1.0 - a0 * a0);
    double phi = 2.0 * M_PI * rng.next();
    double cos_theta = 2.0 * rng.next() - 1.0;
    double sin_theta = std::sqrt(1.0 - cos_theta * cos_theta);
    return Q4{{a0, r_spatial * sin_theta * std::cos(phi), r_spatial * sin_theta * std::sin(phi),
               r_spatial * cos_theta}};
}

// su2_step -- src/heatbath/heatbath.cpp:39-44
inline Q4 su2_step(double beta, const Q4& w, LinkStream& rng) {
    double k = std::sqrt(w.a[0] * w.a[0] + w.a[1] * w.a[1] + w.a[2] * w.a[2] + w.a[3] * w.a[3]);
    Q4 v{{w.a[0] / k, w.a[1] / k, w.a[2] / k, w.a[3] / k}};
    Q4 x = generate_su2_kp(beta, k, rng);
    return qmult(x, qadj(v));
}

// ---------------------------------------------------------------- stencils
// compute_staple -- src/gauge/GaugeField.cpp:74-97
inline M3 staple(const double* U, const Lat& lat, long x, int mu) {
    M3 A = zero3();
    long xmu = lat.neigh(x, mu, +1);
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        long xnu = lat.neigh(x, nu, +1);
        M3 U0 = load(U, xmu, nu), U1 = load(U, xnu, mu), U2 = load(U, x, nu);
        A = add(A, mul(U0, adj(mul(U2, U1))));
        long xmunu = lat.neigh(xmu, nu, -1);
        long xmnu = lat.neigh(x, nu, -1);
        M3 V0 = load(U, xmunu, nu), V1 = load(U, xmnu, mu), V2 = load(U, xmnu, nu);
        A = add(A, mul(adj(mul(V1, V0)), V2));
    }
    return A;
}

// hit -- src/heatbath/heatbath_mpi.cpp:10-33.  refcost: recompute the staple as the reference does.
inline void hb_link(double* U, const Lat& lat, long x, int mu, double beta, int n_hits, LinkStream& rng,
                    bool refcost) {
    M3 A = staple(U, lat, x, mu);
    for (int h = 0; h < n_hits; h++) {
        if (refcost && h > 0) A = staple(U, lat, x, mu);  // identical value: A does not contain U(x,mu)
        M3 Ux = load(U, x, mu);
        M3 W = mul(Ux, A);
        Q4 wq = su2_to_quaternion(W(0, 0), W(0, 1), W(1, 0), W(1, 1));
        Q4 r = su2_step(beta, wq, rng);
        Ux = mul(su2_quaternion_to_su3(r, 0, 1), Ux);

        W = mul(Ux, A);
        wq = su2_to_quaternion(W(1, 1), W(1, 2), W(2, 1), W(2, 2));
        r = su2_step(beta, wq, rng);
        Ux = mul(su2_quaternion_to_su3(r, 1, 2), Ux);

        W = mul(Ux, A);
        wq = su2_to_quaternion(W(0, 0), W(0, 2), W(2, 0), W(2, 2));
        r = su2_step(beta, wq, rng);
        Ux = mul(su2_quaternion_to_su3(r, 0, 2), Ux);
        store(U, x, mu, Ux);
    }
}

void hb_subsweep_impl(double* U, const Lat& lat, double beta, int n_hits, uint64_t seed, uint32_t sweep,
                      int parity, int mu, bool refcost) {
#pragma omp parallel for schedule(static)
    for (long x = 0; x < lat.V; x++) {
        if (lat.parity(x) != parity) continue;
        LinkStream rng(seed, (uint32_t)(x * 4 + mu), sweep, TAG_HB);
        hb_link(U, lat, x, mu, beta, n_hits, rng, refcost);
    }
}

// Deterministic sum of per-site values: fixed t-slice partition, summed in order.
template <class F>
void site_sums(const Lat& lat, int nval, double* out, F f) {
    int Lt = lat.L[3];
    long slice = lat.V / Lt;
    std::vector<double> part((size_t)Lt * nval, 0.0);
#pragma omp parallel for schedule(static)
    for (int t = 0; t < Lt; t++) {
        double acc[4] = {0, 0, 0, 0};
        for (long s = t * slice; s < (t + 1) * slice; s++) {
            double v[4];
            f(s, v);
            for (int k = 0; k < nval; k++) acc[k] += v[k];
        }
        for (int k = 0; k < nval; k++) part[(size_t)t * nval + k] = acc[k];
    }
    for (int k = 0; k < nval; k++) {
        double a = 0.0;
        for (int t = 0; t < Lt; t++) a += part[(size_t)t * nval + k];
        out[k] = a;
    }
}

// plaquette at one site -- src/observables/observables_mpi.cpp:11-35
inline double site_plaquette(const double* U, const Lat& lat, long x) {
    double sum = 0.0;
    for (int mu = 0; mu < 4; mu++)
        for (int nu = mu + 1; nu < 4; nu++) {
            M3 U1 = load(U, x, mu);
            M3 U2 = load(U, lat.neigh(x, mu, +1), nu);
            M3 U3 = adj(load(U, lat.neigh(x, nu, +1), mu));
            M3 U4 = adj(load(U, x, nu));
            sum += trace(mul(mul(mul(U1, U2), U3), U4)).re / 3.0;
        }
    return sum;
}

// clover_site -- src/observables/observables_mpi.cpp:66-90
inline M3 clover_site(const double* U, const Lat& lat, long x, int mu, int nu) {
    long xpmu = lat.neigh(x, mu, +1), xpnu = lat.neigh(x, nu, +1);
    long xmmu = lat.neigh(x, mu, -1), xmnu = lat.neigh(x, nu, -1);
    long xmmupnu = lat.neigh(xmmu, nu, +1), xmmumnu = lat.neigh(xmmu, nu, -1);
    long xpmumnu = lat.neigh(xpmu, nu, -1);
    M3 C = zero3();
    C = add(C, mul(mul(mul(load(U, x, mu), load(U, xpmu, nu)), adj(load(U, xpnu, mu))), adj(load(U, x, nu))));
    C = add(C, mul(mul(mul(load(U, x, nu), adj(load(U, xmmupnu, mu))), adj(load(U, xmmu, nu))),
                   load(U, xmmu, mu)));
    C = add(C, mul(mul(mul(adj(load(U, xmmu, mu)), adj(load(U, xmmumnu, nu))), load(U, xmmumnu, mu)),
                   load(U, xmnu, nu)));
    C = add(C, mul(mul(mul(adj(load(U, xmnu, nu)), load(U, xmnu, mu)), load(U, xpmumnu, nu)),
                   adj(load(U, x, mu))));
    M3 F = sub(C, adj(C));
    return scale(0.125, F);
}

inline double sqnorm(const M3& a) {
    double s = 0.0;
    for (int k = 0; k < 9; k++) s += a.m[k].re * a.m[k].re + a.m[k].im * a.m[k].im;
    return s;
}

// local_q_e_clover -- src/observables/observables_mpi.cpp:93-112
inline void local_q_e(const double* U, const Lat& lat, long x, double* q, double* e) {
    M3 F01 = clover_site(U, lat, x, 0, 1), F02 = clover_site(U, lat, x, 0, 2);
    M3 F03 = clover_site(U, lat, x, 0, 3), F12 = clover_site(U, lat, x, 1, 2);
    M3 F13 = clover_site(U, lat, x, 1, 3), F23 = clover_site(U, lat, x, 2, 3);
    double qq = trace(mul(F01, F23)).re - trace(mul(F02, F13)).re + trace(mul(F03, F12)).re;
    double el = 0.5 * (sqnorm(F01) + sqnorm(F02) + sqnorm(F03) + sqnorm(F12) + sqnorm(F13) + sqnorm(F23));
    *q = qq * (1.0 / (4.0 * M_PI * M_PI));
    *e = el;
}

// ---------------------------------------------------------------- Wilson flow
// GradientFlow state (src/flow/gradient_flow.h:11-27) on a periodic lattice.
struct Flow {
    const Lat& lat;
    double eps;
    double* Uc;
    std::vector<double> F0, F1;
    Flow(const Lat& l, double e, double* U) : lat(l), eps(e), Uc(U), F0(l.V * 72), F1(l.V * 72) {}
    // compute_force -- gradient_flow.cpp:17-37
    void compute_force(int i) {
        double* F = (i == 0) ? F0.data() : F1.data();
#pragma omp parallel for schedule(static)
        for (long x = 0; x < lat.V; x++)
            for (int mu = 0; mu < 4; mu++) {
                M3 A = staple(Uc, lat, x, mu);
                M3 tmp = mul(scale(-1.0, load(Uc, x, mu)), A);
                proj_lie_su3(tmp);
                store(F, x, mu, tmp);
            }
    }
    // compute_w1 -- gradient_flow.cpp:40-57
    void w1() {
#pragma omp parallel for schedule(static)
        for (long x = 0; x < lat.V; x++)
            for (int mu = 0; mu < 4; mu++)
                store(Uc, x, mu, mul(exp_su3_luscher(load(F0.data(), x, mu), 0.25 * eps), load(Uc, x, mu)));
    }
    // compute_w2 -- gradient_flow.cpp:60-79
    void w2() {
#pragma omp parallel for schedule(static)
        for (long x = 0; x < lat.V; x++)
            for (int mu = 0; mu < 4; mu++) {
                M3 Z = sub(scale((8.0 / 9.0) * eps, load(F1.data(), x, mu)),
                           scale((17.0 / 36.0) * eps, load(F0.data(), x, mu)));
                store(Uc, x, mu, mul(exp_su3_luscher(Z, 1.0), load(Uc, x, mu)));
            }
    }
    // replace_force_0 -- gradient_flow.cpp:82-99
    void replace_force_0() {
#pragma omp parallel for schedule(static)
        for (long x = 0; x < lat.V; x++)
            for (int mu = 0; mu < 4; mu++) {
                M3 t = sub(scale(8.0 / 9.0, load(F1.data(), x, mu)), scale(17.0 / 36.0, load(F0.data(), x, mu)));
                store(F0.data(), x, mu, t);
            }
    }
    // compute_w3 -- gradient_flow.cpp:102-121
    void w3() {
#pragma omp parallel for schedule(static)
        for (long x = 0; x < lat.V; x++)
            for (int mu = 0; mu < 4; mu++) {
                M3 Z = sub(scale(0.75 * eps, load(F1.data(), x, mu)), scale(eps, load(F0.data(), x, mu)));
                store(Uc, x, mu, mul(exp_su3_luscher(Z, 1.0), load(Uc, x, mu)));
            }
    }
    // rk3_step -- gradient_flow.cpp:124-135 (halo exchanges are no-ops on a periodic lattice)
    void rk3_step() {
        compute_force(0);
        w1();
        compute_force(1);
        w2();
        replace_force_0();
        compute_force(1);
        w3();
    }
};

void clover_totals(const double* U, const Lat& lat, double* Q, double* E) {
    double out[2];
    site_sums(lat, 2, out, [&](long s, double* v) { local_q_e(U, lat, s, &v[0], &v[1]); });
    *Q = out[0];
    *E = out[1] / (double)lat.V;
}

int g_threads = 0;
struct ThreadScope {
    int prev;
    ThreadScope() : prev(omp_get_max_threads()) {
        if (g_threads > 0) omp_set_num_threads(g_threads);
    }
    ~ThreadScope() { omp_set_num_threads(prev); }
};

}  // namespace

// ====================================================================== C API
extern "C" {

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox(ctr, key, out); }

void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

void orc_exp_su3_luscher(const double* Z, double coeff, double* out) {
    M3 z;
    std::memcpy(z.m, Z, sizeof(z.m));
    M3 r = exp_su3_luscher(z, coeff);
    std::memcpy(out, r.m, sizeof(r.m));
}

void orc_proj_lie_su3(double* A) {
    M3 a;
    std::memcpy(a.m, A, sizeof(a.m));
    proj_lie_su3(a);
    std::memcpy(A, a.m, sizeof(a.m));
}

void orc_projection_su3(double* U) {
    M3 a;
    std::memcpy(a.m, U, sizeof(a.m));
    projection_su3(a);
    std::memcpy(U, a.m, sizeof(a.m));
}

// cold_start -- GaugeField.cpp:23-33
void orc_cold_start(double* U, const int L[4]) {
    ThreadScope ts;
    Lat lat(L);
    M3 I = ident3();
#pragma omp parallel for schedule(static)
    for (long x = 0; x < lat.V; x++)
        for (int mu = 0; mu < 4; mu++) store(U, x, mu, I);
}

// hot_start -- GaugeField.cpp:10-20 with a Haar SU(3) generator of our own: two complex
// Gaussian columns (Box-Muller from the link's Philox stream) made orthonormal and
// completed exactly as projection_su3 does (GaugeField.cpp:36-58).
void orc_hot_start(double* U, const int L[4], uint64_t seed) {
    ThreadScope ts;
    Lat lat(L);
#pragma omp parallel for schedule(static)
    for (long x = 0; x < lat.V; x++)
        for (int mu = 0; mu < 4; mu++) {
            LinkStream rng(seed, (uint32_t)(x * 4 + mu), 0u, TAG_HOT);
            double g[12];
            for (int k = 0; k < 12; k += 2) {
                double u1 = rng.next(), u2 = rng.next();
                double r = std::sqrt(-2.0 * std::log(1.0 - u1));
                double ph = 2.0 * M_PI * u2;
                g[k] = r * std::cos(ph);
                g[k + 1] = r * std::sin(ph);
            }
            M3 m = zero3();
            for (int i = 0; i < 3; i++) {
                m(i, 0) = cx(g[2 * i], g[2 * i + 1]);
                m(i, 1) = cx(g[6 + 2 * i], g[6 + 2 * i + 1]);
            }
            projection_su3(m);
            store(U, x, mu, m);
        }
}

void orc_staple_field(const double* U, const int L[4], int mu, double* out) {
    ThreadScope ts;
    Lat lat(L);
#pragma omp parallel for schedule(static)
    for (long x = 0; x < lat.V; x++) {
        M3 A = staple(U, lat, x, mu);
        std::memcpy(out + x * 18, A.m, sizeof(A.m));
    }
}

// mean_plaquette_global -- observables_mpi.cpp:39-48 (single rank: size = 1)
double orc_plaquette(const double* U, const int L[4]) {
    ThreadScope ts;
    Lat lat(L);
    double s;
    site_sums(lat, 1, &s, [&](long x, double* v) { v[0] = site_plaquette(U, lat, x); });
    return s / (6.0 * (double)lat.V);
}

// topo_q_e_clover_global -- observables_mpi.cpp:136-156 (single rank)
void orc_clover_qe(const double* U, const int L[4], double* Q, double* E) {
    ThreadScope ts;
    Lat lat(L);
    clover_totals(U, lat, Q, E);
}

void orc_clover_qe_density(const double* U, const int L[4], double* q, double* e) {
    ThreadScope ts;
    Lat lat(L);
#pragma omp parallel for schedule(static)
    for (long x = 0; x < lat.V; x++) local_q_e(U, lat, x, &q[x], &e[x]);
}

void orc_flow_rk3(double* U, const int L[4], double eps, int n) {
    ThreadScope ts;
    Lat lat(L);
    Flow f(lat, eps, U);
    for (int i = 0; i < n; i++) f.rk3_step();
}

// topo_charge_flowed -- observables_mpi.cpp:159-186
void orc_flow_measure(const double* U, const int L[4], double eps, int n_steps, int n_rk, double* tQE) {
    ThreadScope ts;
    Lat lat(L);
    std::vector<double> Uc(U, U + lat.V * 72);
    Flow f(lat, eps, Uc.data());
    double t = 0.0;
    for (int step = 0; step < n_steps; step++) {
        double Q, E;
        clover_totals(Uc.data(), lat, &Q, &E);
        tQE[3 * step] = t;
        tQE[3 * step + 1] = Q;
        tQE[3 * step + 2] = E;
        if (step != n_steps - 1) {
            for (int k = 0; k < n_rk; k++) {
                f.rk3_step();
                t += eps;
            }
        }
    }
}

void orc_hb_subsweep(double* U, const int L[4], double beta, int n_hits, uint64_t seed, uint32_t sweep,
                     int parity, int mu) {
    ThreadScope ts;
    Lat lat(L);
    hb_subsweep_impl(U, lat, beta, n_hits, seed, sweep, parity, mu, false);
}

void orc_hb_subsweep_refcost(double* U, const int L[4], double beta, int n_hits, uint64_t seed, uint32_t sweep,
                             int parity, int mu) {
    ThreadScope ts;
    Lat lat(L);
    hb_subsweep_impl(U, lat, beta, n_hits, seed, sweep, parity, mu, true);
}

void orc_hb_sweep(double* U, const int L[4], double beta, int n_hits, uint64_t seed, uint32_t sweep) {
    ThreadScope ts;
    Lat lat(L);
    for (int p = 0; p < 2; p++)
        for (int mu = 0; mu < 4; mu++) hb_subsweep_impl(U, lat, beta, n_hits, seed, sweep, p, mu, false);
}

void orc_hb_sweep_refcost(double* U, const int L[4], double beta, int n_hits, uint64_t seed, uint32_t sweep) {
    ThreadScope ts;
    Lat lat(L);
    for (int p = 0; p < 2; p++)
        for (int mu = 0; mu < 4; mu++) hb_subsweep_impl(U, lat, beta, n_hits, seed, sweep, p, mu, true);
}

// shift_field -- Shift.cpp:109-160: after the shift, site x holds what x - s held.
void orc_shift(double* U, const int L[4], const int s[4]) {
    ThreadScope ts;
    Lat lat(L);
    std::vector<double> src(U, U + lat.V * 72);
#pragma omp parallel for schedule(static)
    for (long x = 0; x < lat.V; x++) {
        int c[4];
        lat.coords(x, c);
        for (int d = 0; d < 4; d++) {
            int sd = s[d] % lat.L[d];
            if (sd < 0) sd += lat.L[d];
            c[d] = (c[d] - sd + lat.L[d]) % lat.L[d];
        }
        long y = lat.index(c);
        std::memcpy(U + x * 72, src.data() + y * 72, 72 * sizeof(double));
    }
}

// random_shift draw semantics -- Shift.cpp:163-176: four integers uniform in [0, n-1].
void orc_random_shift_draw(uint64_t seed, uint64_t idx, const int L[4], int max_shift, int s_out[4]) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t ctr[4] = {0u, (uint32_t)idx, (uint32_t)(idx >> 32), TAG_SHIFT};
    uint32_t o[4];
    philox(ctr, key, o);
    for (int d = 0; d < 4; d++) {
        uint32_t n = (uint32_t)(max_shift > 0 ? max_shift : L[d]);
        s_out[d] = (int)(((uint64_t)o[d] * n) >> 32);
    }
}

// project_field_su3 -- GaugeField.cpp:61-71
void orc_reunitarize(double* U, const int L[4]) {
    ThreadScope ts;
    Lat lat(L);
#pragma omp parallel for schedule(static)
    for (long x = 0; x < lat.V; x++)
        for (int mu = 0; mu < 4; mu++) {
            M3 m = load(U, x, mu);
            projection_su3(m);
            store(U, x, mu, m);
        }
}

// unitarity error ||U U^dag - 1||_F -- src/bin/test.cpp:58-72
void orc_unitarity(const double* U, const int L[4], double* max_err, double* mean_err) {
    ThreadScope ts;
    Lat lat(L);
    double mx = 0.0, sum = 0.0;
#pragma omp parallel for schedule(static) reduction(max : mx) reduction(+ : sum)
    for (long x = 0; x < lat.V; x++)
        for (int mu = 0; mu < 4; mu++) {
            M3 u = load(U, x, mu);
            M3 D = sub(mul(u, adj(u)), ident3());
            double err = std::sqrt(trace(mul(adj(D), D)).re);
            if (err > mx) mx = err;
            sum += err;
        }
    *max_err = mx;
    *mean_err = sum / (4.0 * (double)lat.V);
}

}  // extern "C"
