// qcb_kernels.cuh -- sm_100a kernels of the gauge-field hot path.
//
// Every kernel is templated on the storage real type R (double / float) and on the
// number of stored complex entries per link NE (9 = 18 reals, 6 = 12 reals).
#pragma once
#include <stdint.h>

#include "qcb_field.cuh"

namespace qcb {

constexpr double kPi = 3.14159265358979323846;

// Device error flags (bit mask written by kernels, read by the host after a sync).
enum : int { DERR_KP_CAP = 1, DERR_KP_SCALE = 2, DERR_BULK_WAIT = 4 };

// ------------------------------------------------------------------ bulk copies into shared memory
// One-shot mbarrier-tracked bulk copies (the TMA engine's cp.async.bulk, global -> this CTA's shared
// memory, no multicast).  Addresses 16-byte aligned, sizes multiples of 16 bytes.
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst), b = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
                 "l"(src), "r"(bytes), "r"(b)
                 : "memory");
}
// Waits for phase `phase` of the barrier, at most max_tries polls (each poll may suspend the thread
// for a bounded, hardware-chosen time); false if the copies did not land in that time.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase, int max_tries) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    for (int i = 0; i < max_tries; i++) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(a), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// byte reversal of a double (ILDG files are big-endian, src/io/ildg.cpp:25-32)
__device__ __forceinline__ double bswap_f64(double x) {
    unsigned long long v = (unsigned long long)__double_as_longlong(x);
    unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
    unsigned long long r = ((unsigned long long)__byte_perm(lo, 0u, 0x0123u) << 32) | __byte_perm(hi, 0u, 0x0123u);
    return __longlong_as_double((long long)r);
}

// ------------------------------------------------------------------ staple
// compute_staple (src/gauge/GaugeField.cpp:74-97):
//   A = sum_{nu != mu} U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag + U_nu(x+mu-nu)^dag U_mu(x-nu)^dag U_nu(x-nu)
// x has parity `par`; x+-nu and x+mu have parity 1-par; x+mu-nu has parity `par`.
template <typename R, int NE, int MU, bool RO>
__device__ __forceinline__ M3<R> staple(const Geom& g, const LinkField<R, NE>& U, const int c[4], int lex,
                                        int par) {
    M3<R> A;
    set_zero(A);
    const int opp = par ^ 1;
    const int xmu = step_up(g, lex, c[MU], MU);
#pragma unroll
    for (int nu = 0; nu < 4; nu++) {
        if (nu == MU) continue;
        const int xnu = step_up(g, lex, c[nu], nu);
        const int xmnu = step_dn(g, lex, c[nu], nu);
        const int xmumnu = step_dn(g, xmu, c[nu], nu);
        {
            M3<R> a = RO ? U.load_ro(nu, opp, xmu >> 1) : U.load(nu, opp, xmu >> 1);
            M3<R> b = RO ? U.load_ro(MU, opp, xnu >> 1) : U.load(MU, opp, xnu >> 1);
            M3<R> t = mul_na(a, b);
            M3<R> d = RO ? U.load_ro(nu, par, lex >> 1) : U.load(nu, par, lex >> 1);
            acc_na(A, t, d);
        }
        {
            M3<R> v1 = RO ? U.load_ro(MU, opp, xmnu >> 1) : U.load(MU, opp, xmnu >> 1);
            M3<R> v0 = RO ? U.load_ro(nu, par, xmumnu >> 1) : U.load(nu, par, xmumnu >> 1);
            M3<R> t = mul_nn(v1, v0);
            M3<R> v2 = RO ? U.load_ro(nu, opp, xmnu >> 1) : U.load(nu, opp, xmnu >> 1);
            acc_an(A, t, v2);
        }
    }
    return A;
}

// Same staple with a runtime direction and a rolled nu loop: one code path for all four
// directions (a single kernel then serves every link class without four unrolled copies
// competing for the instruction cache).  The nu order is the reference's (ascending, skip mu).
template <typename R, int NE>
__device__ __forceinline__ M3<R> staple_rt(const Geom& g, const LinkField<R, NE>& U, const int c[4], int lex,
                                           int par, int mu) {
    M3<R> A;
    set_zero(A);
    const int opp = par ^ 1;
    const Steps st = make_steps(g, c);
    const int xmu = lex + sel4(st.up, mu);
#pragma unroll 1
    for (int k = 0; k < 3; k++) {
        const int nu = k < mu ? k : k + 1;
        const int dnu = sel4(st.dn, nu);
        const int xnu = lex + sel4(st.up, nu);
        const int xmnu = lex + dnu;
        const int xmumnu = xmu + dnu;  // x+mu has the same nu coordinate as x
        {
            M3<R> a = U.load_ro(nu, opp, xmu >> 1);
            M3<R> b = U.load_ro(mu, opp, xnu >> 1);
            M3<R> t = mul_na(a, b);
            M3<R> d = U.load_ro(nu, par, lex >> 1);
            acc_na(A, t, d);
        }
        {
            M3<R> v1 = U.load_ro(mu, opp, xmnu >> 1);
            M3<R> v0 = U.load_ro(nu, par, xmumnu >> 1);
            M3<R> t = mul_nn(v1, v0);
            M3<R> v2 = U.load_ro(nu, opp, xmnu >> 1);
            acc_an(A, t, v2);
        }
    }
    return A;
}

// FP32 staple with two-row products.  Every staple is a product of three SU(3) links, so it is
// itself in SU(3) up to rounding: only its first two rows are formed by products and the third
// is the conjugate cross product r2 = conj(r0 x r1).  Forward staple a b^dag d^dag
// (a = U_nu(x+mu), b = U_mu(x+nu), d = U_nu(x)): rows 0-1 of a b^dag, then of (a b^dag) d^dag.
// Backward staple t^dag v2 with t = v1 v0 (v1 = U_mu(x-nu), v0 = U_nu(x+mu-nu), v2 = U_nu(x-nu)):
// rows 0-1 of t^dag need columns 0-1 of t only.  That is 42 instead of 54 complex
// multiply-adds a staple.  The rebuilt row differs from the explicit product by the
// links' distance from SU(3), which in FP32 storage is the FP32 rounding level (~1e-7).
template <typename R, int NE>
__device__ __forceinline__ M3<R> staple_rt_rows(const Geom& g, const LinkField<R, NE>& U, const int c[4],
                                                int lex, int par, int mu) {
    M3<R> A;
    set_zero(A);
    const int opp = par ^ 1;
    const Steps st = make_steps(g, c);
    const int xmu = lex + sel4(st.up, mu);
#pragma unroll 1
    for (int k = 0; k < 3; k++) {
        const int nu = k < mu ? k : k + 1;
        const int dnu = sel4(st.dn, nu);
        const int xnu = lex + sel4(st.up, nu);
        const int xmnu = lex + dnu;
        const int xmumnu = xmu + dnu;  // x+mu has the same nu coordinate as x
        {
            const M3<R> a = U.load_ro(nu, opp, xmu >> 1);
            const M3<R> b = U.load_ro(mu, opp, xnu >> 1);
            Cx<R> t[2][3], s[2][3];
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    t[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac_nc(t[i][j], a(i, q), b(j, q));
                }
            const M3<R> d = U.load_ro(nu, par, lex >> 1);
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    s[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac_nc(s[i][j], t[i][q], d(j, q));
                    A(i, j) = A(i, j) + s[i][j];
                }
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                A(2, j) = A(2, j) + conj_cross(s[0][j1], s[1][j2], s[0][j2], s[1][j1]);
            }
        }
        {
            const M3<R> v1 = U.load_ro(mu, opp, xmnu >> 1);
            const M3<R> v0 = U.load_ro(nu, par, xmumnu >> 1);
            Cx<R> t[3][2], s[2][3];
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    t[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac(t[i][j], v1(i, q), v0(q, j));
                }
            const M3<R> v2 = U.load_ro(nu, opp, xmnu >> 1);
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    s[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac_cn(s[i][j], t[q][i], v2(q, j));
                    A(i, j) = A(i, j) + s[i][j];
                }
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                A(2, j) = A(2, j) + conj_cross(s[0][j1], s[1][j2], s[0][j2], s[1][j1]);
            }
        }
    }
    return A;
}

// ------------------------------------------------------------------ clover halves from the force's staples
// The clover sum C of plane (mu, nu) at site x (clover_site, observables_mpi.cpp:66-90) enters the
// observables only through acc(C): o_ij = C_ij - conj(C_ji) (i < j) and d_i = Im C_ii, which is
// linear and odd under the adjoint.  With D(y) = S_f(y) - S_b(y), the forward minus the backward
// staple of link (y, mu) in plane nu (the two terms compute_staple sums for that plane),
//   leaves 1 + 4 of x:  acc(U_mu(x) D(x)),      leaves 2 + 3 of x:  acc(D(x - mu) U_mu(x - mu)),
// since leaf 1 = U_mu(x) S_f(x), leaf 4 = (U_mu(x) S_b(x))^dag, leaf 2 = S_f(x-mu) U_mu(x-mu) and
// leaf 3 = (S_b(x-mu) U_mu(x-mu))^dag, and acc(X^dag) = -acc(X).  Stage 1 of an RK3 step forms S_f and
// S_b of every link for its force, so with two more products a plane (U D and D U) it yields the
// clover of its input configuration: the link (y, mu) writes the half for leaves 1 + 4 of y and the
// half for leaves 2 + 3 of y + mu, and k_clover_halves adds the two halves of each site.  From the
// nu links, plane (mu, nu) appears with the orientation reversed and both halves change sign.
// Each plane is handled by the links of one direction (two planes at most a direction):
//   plane 01 -> 0, 02 -> 2, 03 -> 3, 12 -> 1, 13 -> 3, 23 -> 2.
__host__ __device__ __forceinline__ int plane_index(int a, int b) {  // a < b: 01 02 03 12 13 23
    return a == 0 ? b - 1 : (a == 1 ? b + 1 : 5);
}
__host__ __device__ __forceinline__ int plane_owner(int p) { return (0x231320 >> (4 * p)) & 0xF; }

// The halves of every (plane, site): nine reals (o01, o02, o12 as re/im pairs, then d0, d1, d2) for
// half 0 (leaves 1 + 4) and half 1 (leaves 2 + 3) of each plane, and Re Tr of leaf 1 (the plaquette
// trace) of each plane; reals at p[k * V + site], site = parity * Vh + h.
template <typename R>
struct HalfClovers {
    R* p;
    int64_t V;
    // offset of real k of a site; the checked build validates (k, site) as it does link indices
    // (kind 2) and redirects a bad one to real 0 of site 0
    __device__ __forceinline__ int64_t at(int k, int64_t site) const {
#if defined(QCB_CHECKED) && defined(__CUDA_ARCH__)
        if (!((unsigned)k < (unsigned)(6 * 2 * 9 + 6) && site >= 0 && site < V)) {
            note_oob(2, k, site >= V ? 1 : 0, site);
            k = 0;
            site = 0;
        }
#endif
        return (int64_t)k * V + site;
    }
    __device__ __forceinline__ void put_half(int plane, int half, int64_t site, const R v[9], R sign) const {
#pragma unroll
        for (int k = 0; k < 9; k++) p[at((plane * 2 + half) * 9 + k, site)] = sign * v[k];
    }
    __device__ __forceinline__ void put_plaq(int plane, int64_t site, R tr) const { p[at(108 + plane, site)] = tr; }
    __device__ __forceinline__ R half(int plane, int half, int k, int64_t site) const {
        return p[at((plane * 2 + half) * 9 + k, site)];
    }
    __device__ __forceinline__ R plaq(int plane, int64_t site) const { return p[at(108 + plane, site)]; }
};

// acc(A B) for full 3x3 A, B: the six off-diagonal entries of A B and the imaginary parts of its
// diagonal, in the order of HalfClovers.
template <typename R>
__device__ __forceinline__ void acc_product(const M3<R>& A, const M3<R>& B, R out[9]) {
    Cx<R> m[3][3];
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if (i == j) continue;
            m[i][j] = mkc<R>(0, 0);
#pragma unroll
            for (int q = 0; q < 3; q++) cmac(m[i][j], A(i, q), B(q, j));
        }
    const int I[3] = {0, 0, 1}, J[3] = {1, 2, 2};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        out[2 * k] = m[I[k]][J[k]].re - m[J[k]][I[k]].re;
        out[2 * k + 1] = m[I[k]][J[k]].im + m[J[k]][I[k]].im;
    }
#pragma unroll
    for (int i = 0; i < 3; i++) {
        R im = R(0);
#pragma unroll
        for (int q = 0; q < 3; q++) im = fma(A(i, q).re, B(q, i).im, fma(A(i, q).im, B(q, i).re, im));
        out[6 + i] = im;
    }
}

// staple_rt_rows, and for the planes this direction handles the two clover halves and the plaquette
// trace of the link's site (see above).  u is the link U_mu(x) itself.
template <typename R, int NE>
__device__ __forceinline__ M3<R> staple_rt_rows_meas(const Geom& g, const LinkField<R, NE>& U, const int c[4],
                                                     int lex, int par, int mu, const M3<R>& u_in,
                                                     const HalfClovers<R>& H) {
    M3<R> A;
    set_zero(A);
    const int opp = par ^ 1;
    const Steps st = make_steps(g, c);
    const int xmu = lex + sel4(st.up, mu);
    const int64_t site = (int64_t)par * g.Vh + (lex >> 1), site_up = (int64_t)opp * g.Vh + (xmu >> 1);
#pragma unroll 1
    for (int k = 0; k < 3; k++) {
        const int nu = k < mu ? k : k + 1;
        const int plane = mu < nu ? plane_index(mu, nu) : plane_index(nu, mu);
        const bool owned = plane_owner(plane) == mu;
        const int dnu = sel4(st.dn, nu);
        const int xnu = lex + sel4(st.up, nu);
        const int xmnu = lex + dnu;
        const int xmumnu = xmu + dnu;
        M3<R> Sf;
        {
            const M3<R> a = U.load_ro(nu, opp, xmu >> 1);
            const M3<R> b = U.load_ro(mu, opp, xnu >> 1);
            Cx<R> t[2][3];
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    t[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac_nc(t[i][j], a(i, q), b(j, q));
                }
            const M3<R> d = U.load_ro(nu, par, lex >> 1);
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    Cx<R> v = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac_nc(v, t[i][q], d(j, q));
                    Sf(i, j) = v;
                    A(i, j) = A(i, j) + v;
                }
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                Sf(2, j) = conj_cross(Sf(0, j1), Sf(1, j2), Sf(0, j2), Sf(1, j1));
                A(2, j) = A(2, j) + Sf(2, j);
            }
        }
        M3<R> Sb;
        {
            const M3<R> v1 = U.load_ro(mu, opp, xmnu >> 1);
            const M3<R> v0 = U.load_ro(nu, par, xmumnu >> 1);
            Cx<R> t[3][2];
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    t[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac(t[i][j], v1(i, q), v0(q, j));
                }
            const M3<R> v2 = U.load_ro(nu, opp, xmnu >> 1);
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    Cx<R> v = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac_cn(v, t[q][i], v2(q, j));
                    Sb(i, j) = v;
                    A(i, j) = A(i, j) + v;
                }
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                Sb(2, j) = conj_cross(Sb(0, j1), Sb(1, j2), Sb(0, j2), Sb(1, j1));
                A(2, j) = A(2, j) + Sb(2, j);
            }
        }
        if (owned) {
            // FP64: the link is reloaded here (an L1 hit) instead of held across the loop, which
            // lets the kernel run 3 blocks/SM (measured flow 2.73-2.74 against 2.79-2.80 ms a 32^4
            // step); FP32 holds it (no gain from the reload)
            const M3<R> u = (sizeof(R) == 8) ? U.load_ro(mu, par, lex >> 1) : u_in;
            R tr = R(0);
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int q = 0; q < 3; q++) tr = fma(u(i, q).re, Sf(q, i).re, fma(-u(i, q).im, Sf(q, i).im, tr));
            H.put_plaq(plane, site, tr);
            M3<R> D;
#pragma unroll
            for (int e = 0; e < 9; e++) D.e[e] = Sf.e[e] - Sb.e[e];
            const R sign = mu < nu ? R(1) : R(-1);
            R v[9];
            acc_product(u, D, v);
            H.put_half(plane, 0, site, v, sign);
            acc_product(D, u, v);
            H.put_half(plane, 1, site_up, v, sign);
        }
    }
    return A;
}

// -proj_lie(u A) (compute_force, gradient_flow.cpp:17-37) forming only the entries the
// projection reads: the six off-diagonal entries of u A and the imaginary parts of its diagonal.
template <typename R>
__device__ __forceinline__ M3<R> neg_proj_lie_mul(const M3<R>& u, const M3<R>& A) {
    M3<R> m;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if (i == j) {
                R im = R(0);
#pragma unroll
                for (int q = 0; q < 3; q++) im = fma(u(i, q).re, A(q, i).im, fma(u(i, q).im, A(q, i).re, im));
                m(i, i) = mkc<R>(R(0), im);
            } else {
                Cx<R> v = mkc<R>(0, 0);
#pragma unroll
                for (int q = 0; q < 3; q++) cmac(v, u(i, q), A(q, j));
                m(i, j) = v;
            }
        }
    M3<R> F;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            if (i != j) F(i, j) = mkc<R>(R(-0.5) * (m(i, j).re - m(j, i).re), R(-0.5) * (m(i, j).im + m(j, i).im));
    const R tr3 = (m(0, 0).im + m(1, 1).im + m(2, 2).im) / R(3);
#pragma unroll
    for (int i = 0; i < 3; i++) F(i, i) = mkc<R>(R(0), tr3 - m(i, i).im);
    return F;
}

// Launch shapes (measured on B200, 32^4): 128-thread blocks.  Minimum resident blocks per SM:
// heatbath 4 for FP64 (<= 128 registers; 0.206 ms a sub-sweep at N_hits = 2; 3, 5 and 6 blocks
// are slower, 64-thread blocks at 8 per SM within 1%) and 6 for FP32; flow stages 3 for FP64 (<= 168 registers; 4 is no faster) and 6 for FP32
// (<= 80 registers, no spills: 0.36 ms a stage against 0.40 ms at 4 and 0.37 ms at 8).
#ifndef QCB_HB_THREADS
#define QCB_HB_THREADS 128
#endif
#ifndef QCB_HB_MINB
#define QCB_HB_MINB(R) (sizeof(R) == 8 ? 4 : 6)
#endif
#ifndef QCB_HB_BULK_LINKS
#define QCB_HB_BULK_LINKS 0
#endif
#ifndef QCB_FLOW_THREADS
#define QCB_FLOW_THREADS 128
#endif
// shared (tile) flow stage of the server's small requests: FP32 at 5 blocks/SM (102 registers, no
// spills; 24 resident 16^4 requests x 300 steps 0.83-0.90 s against 0.91-0.95 s at 6)
#ifndef QCB_FLOW_MINB
#define QCB_FLOW_MINB(R) (sizeof(R) == 8 ? 3 : 5)
#endif
// Clover kernels: 2 resident blocks per SM for FP64, 4 for FP32 (32^4 clover pass 1.02 ms FP64 and
// 0.49 ms FP32 against 1.24 ms and 0.69 ms at 3 and 6).
#ifndef QCB_CLOVER_MINB
#define QCB_CLOVER_MINB(R) (sizeof(R) == 8 ? 2 : 4)
#endif
// single-lattice flow stage launch shape (the tiled kernels keep QCB_FLOW_THREADS = TILE)
#ifndef QCB_FLOW1_THREADS
#define QCB_FLOW1_THREADS QCB_FLOW_THREADS
#endif
#ifndef QCB_FLOW1_MINB
#define QCB_FLOW1_MINB(R) (sizeof(R) == 8 ? 3 : 6)
#endif
// stage 1 with the clover halves: the forward staple is held until the backward one is formed
// (FP64 3 blocks/SM with the link reloaded for the halves, no spills; FP32 4)
#ifndef QCB_FLOW_MEAS_MINB
#define QCB_FLOW_MEAS_MINB(R) (sizeof(R) == 8 ? 3 : 4)
#endif
#ifndef QCB_FLOW_RTMU
#define QCB_FLOW_RTMU 1
#endif
// FP64 flow stages and clover leaves with two-row products (third row rebuilt as conj(r0 x r1)),
// as in FP32.  The rebuilt rows differ from explicit products by the links' distance from SU(3),
// ~1e-15 in FP64, inside the 1e-12 parity bound; the flow stage runs 8% faster.
#ifndef QCB_FLOW64_ROWS
#define QCB_FLOW64_ROWS 1
#endif
#ifndef QCB_CLOVER64_ROWS
#define QCB_CLOVER64_ROWS 1
#endif

// ------------------------------------------------------------------ heatbath
struct Quat {
    double a0, a1, a2, a3;
};

// Heatbath draws ahead of use.  A subgroup update consumes Philox calls n, n+1 per Kennedy-Pendleton
// attempt and one call for (u_phi, u_cos) after the accepted attempt, so the stream position is
// even at every subgroup and a subgroup starting at call n needs calls n, n+1 (attempt 0) and
// n+2 (its final draws if attempt 0 is accepted, else attempt 1's first pair).  P, Q, F hold
// those three calls, evaluated together (independent Philox chains) before they are needed.
struct KPDraws {
    uint32_t n;  // first call of the current subgroup
    double2 P, Q, F;
};
__device__ __forceinline__ KPDraws kp_draws_at(const LinkStream& rng, uint32_t n) {
    KPDraws d;
    d.n = n;
    d.P = rng.call(n);
    d.Q = rng.call(n + 1);
    d.F = rng.call(n + 2);
    return d;
}

// generate_su2_kp (src/heatbath/heatbath.cpp:8-36) + su2_step (:39-44), drawing in the
// reference's order: (delta, r1, r2, r3) per Kennedy-Pendleton attempt, then (u_phi, u_cos).
// With c_alpha = -0.75/beta, -0.5/alpha = c_alpha / k (alpha = 2 beta k / 3), so one rsqrt
// gives both v = w/k and the attempt scale.
// The reference loops until acceptance.  Here the loop is capped at KP_MAX_ATTEMPTS = 2^20
// attempts, so that no lane can spin without bound: acceptance falls roughly like alpha^1.5, and
// the cap is reached only for alpha ~ 1e-4 (|w| ~ 1e-5), which the updates of hot and thermalised
// configurations never produce.  On the cap the subgroup element is the identity (the link is left
// unchanged by this subgroup) and the kernel raises DERR_KP_CAP; a zero or non-finite |w| (a
// non-finite or non-negative scale) is rejected up front in the same way and raises DERR_KP_SCALE.
// `d` holds this subgroup's first draws on entry; with `more` set it holds the next subgroup's
// on return (evaluated right after acceptance, alongside the rest of this update).
constexpr int KP_MAX_ATTEMPTS = 1 << 20;
__device__ __forceinline__ Quat su2_step(double c_alpha, Quat w, const LinkStream& rng, KPDraws& d, bool more,
                                         int* err) {
    const double ik = rsqrt(w.a0 * w.a0 + w.a1 * w.a1 + w.a2 * w.a2 + w.a3 * w.a3);  // 1/k
    const Quat v = {w.a0 * ik, w.a1 * ik, w.a2 * ik, w.a3 * ik};
    const double m05a = c_alpha * ik;  // -0.5 / alpha
    double a0 = 1.0;
    bool ok = false;
    const int cap = (m05a < 0.0 && isfinite(m05a)) ? KP_MAX_ATTEMPTS : 0;
    const uint32_t n = d.n;
    double2 P = d.P, Q = d.Q, F = d.F;
    int it = 0;
    for (; it < cap; it++) {
        const double delta = P.x, r1 = P.y, r2 = Q.x, r3 = Q.y;
        double c = cospi(2.0 * r2);
        double lsq = __dmul_rn(m05a, __dadd_rn(log(r1), __dmul_rn(__dmul_rn(c, c), log(r3))));
        if (__dmul_rn(delta, delta) <= __dadd_rn(1.0, -lsq)) {
            a0 = __dadd_rn(1.0, -__dmul_rn(2.0, lsq));
            ok = true;
            break;
        }
        // attempt it + 1 uses calls n + 2it + 2 (= F) and n + 2it + 3
        P = F;
        Q = rng.call(n + 2u * (uint32_t)it + 3u);
        F = rng.call(n + 2u * (uint32_t)it + 4u);
    }
    // accepted at attempt it: calls n .. n + 2it + 2 are used; failed: 2 cap calls, no final draws
    const uint32_t n_next = ok ? n + 2u * (uint32_t)it + 3u : n + 2u * (uint32_t)cap;
    if (more) d = kp_draws_at(rng, n_next);
    if (!ok) {
        atomicOr(err, cap > 0 ? (int)DERR_KP_CAP : (int)DERR_KP_SCALE);
        return Quat{1.0, 0.0, 0.0, 0.0};
    }
    const double rs = sqrt(1.0 - a0 * a0);
    const double uphi = F.x;
    const double cos_t = 2.0 * F.y - 1.0;
    const double sin_t = sqrt(1.0 - cos_t * cos_t);
    double sp, cp;
    sincospi(2.0 * uphi, &sp, &cp);
    const Quat x = {a0, rs * sin_t * cp, rs * sin_t * sp, rs * cos_t};
    // mult(x, adj(v))  (src/su3/utils.cpp:53-63)
    return Quat{x.a0 * v.a0 + x.a1 * v.a1 + x.a2 * v.a2 + x.a3 * v.a3,
                -x.a0 * v.a1 + x.a1 * v.a0 - x.a2 * v.a3 + x.a3 * v.a2,
                -x.a0 * v.a2 + x.a1 * v.a3 + x.a2 * v.a0 - x.a3 * v.a1,
                -x.a0 * v.a3 - x.a1 * v.a2 + x.a2 * v.a1 + x.a3 * v.a0};
}

// One Cabibbo-Marinari subgroup update of u in place (src/heatbath/heatbath_mpi.cpp:14-32):
// w = quaternion of the (I,J) block of W = u*A, r = su2_step(w), u <- embed_{IJ}(r) * u.
template <typename R, int I, int J, typename AM>
__device__ __forceinline__ void cm_subgroup(M3<R>& u, const AM& A, double c_alpha, const LinkStream& rng, KPDraws& d,
                                            bool more, int* err) {
    Cx<R> wii = mkc<R>(0, 0), wij = mkc<R>(0, 0), wji = mkc<R>(0, 0), wjj = mkc<R>(0, 0);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        cmac(wii, u(I, k), A(k, I));
        cmac(wij, u(I, k), A(k, J));
        cmac(wji, u(J, k), A(k, I));
        cmac(wjj, u(J, k), A(k, J));
    }
    // su2_to_quaternion (src/su3/utils.cpp:47-50)
    Quat w = {((double)wii.re + (double)wjj.re) / 2.0, ((double)wij.im + (double)wji.im) / 2.0,
              ((double)wij.re - (double)wji.re) / 2.0, ((double)wii.im - (double)wjj.im) / 2.0};
    Quat r = su2_step(c_alpha, w, rng, d, more, err);
    // su2_quaternion_to_su3 (src/su3/utils.cpp:33-44) applied from the left
    Cx<R> rii = mkc<R>((R)r.a0, (R)r.a3), rjj = mkc<R>((R)r.a0, (R)-r.a3);
    Cx<R> rij = mkc<R>((R)r.a2, (R)r.a1), rji = mkc<R>((R)-r.a2, (R)r.a1);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        Cx<R> ui = u(I, k), uj = u(J, k);
        Cx<R> ni = rii * ui;
        cmac(ni, rij, uj);
        Cx<R> nj = rji * ui;
        cmac(nj, rjj, uj);
        u(I, k) = ni;
        u(J, k) = nj;
    }
}

// A thread's staple held in shared memory for the hits: element k of the thread's matrix at
// p[k * stride] (p offset by the thread index), so a warp touches 32 consecutive complexes per
// element.  Reads go through ld.shared so the compiler keeps the matrix in shared memory instead
// of forwarding it back into registers; the registers it frees raise the resident warps.
template <typename R>
struct StapleSlot {
    typedef typename V2<R>::T C2;
    C2* p;
    int stride;
    __device__ __forceinline__ void set(int i, int j, Cx<R> v) const {
        const unsigned a = (unsigned)__cvta_generic_to_shared(p + (i * 3 + j) * stride);
        if constexpr (sizeof(R) == 8)
            asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(a), "d"(v.re), "d"(v.im) : "memory");
        else
            asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.re), "f"(v.im) : "memory");
    }
    __device__ __forceinline__ void put(const M3<R>& A) const {
#pragma unroll
        for (int k = 0; k < 9; k++) set(k / 3, k % 3, A.e[k]);
    }
    __device__ __forceinline__ Cx<R> operator()(int i, int j) const {
        const unsigned a = (unsigned)__cvta_generic_to_shared(p + (i * 3 + j) * stride);
        R x, y;
        if constexpr (sizeof(R) == 8)
            asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "r"(a) : "memory");
        else
            asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(x), "=f"(y) : "r"(a) : "memory");
        return mkc<R>(x, y);
    }
    __device__ __forceinline__ M3<R> get() const {
        M3<R> A;
#pragma unroll
        for (int k = 0; k < 9; k++) A.e[k] = (*this)(k / 3, k % 3);
        return A;
    }
};

// staple_rt_rows accumulated into a shared-memory slot instead of registers: each forward or
// backward staple is formed in registers and added to the slot, so the 18-real accumulator does not
// occupy registers across the nu loop.
template <typename R, int NE>
__device__ __forceinline__ void staple_rows_into(const Geom& g, const LinkField<R, NE>& U, const int c[4], int lex,
                                                 int par, int mu, const StapleSlot<R>& S) {
#pragma unroll
    for (int e = 0; e < 9; e++) S.set(e / 3, e % 3, mkc<R>(0, 0));
    const int opp = par ^ 1;
    const Steps st = make_steps(g, c);
    const int xmu = lex + sel4(st.up, mu);
    auto add_rows = [&](const Cx<R> r[2][3]) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            const Cx<R> r2 = conj_cross(r[0][j1], r[1][j2], r[0][j2], r[1][j1]);
            S.set(0, j, S(0, j) + r[0][j]);
            S.set(1, j, S(1, j) + r[1][j]);
            S.set(2, j, S(2, j) + r2);
        }
    };
#pragma unroll 1
    for (int k = 0; k < 3; k++) {
        const int nu = k < mu ? k : k + 1;
        const int dnu = sel4(st.dn, nu);
        const int xnu = lex + sel4(st.up, nu);
        const int xmnu = lex + dnu;
        const int xmumnu = xmu + dnu;
        {
            const M3<R> a = U.load_ro(nu, opp, xmu >> 1);
            const M3<R> b = U.load_ro(mu, opp, xnu >> 1);
            Cx<R> t[2][3], r[2][3];
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    t[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac_nc(t[i][j], a(i, q), b(j, q));
                }
            const M3<R> d = U.load_ro(nu, par, lex >> 1);
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    r[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac_nc(r[i][j], t[i][q], d(j, q));
                }
            add_rows(r);
        }
        {
            const M3<R> v1 = U.load_ro(mu, opp, xmnu >> 1);
            const M3<R> v0 = U.load_ro(nu, par, xmumnu >> 1);
            Cx<R> t[3][2], r[2][3];
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    t[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac(t[i][j], v1(i, q), v0(q, j));
                }
            const M3<R> v2 = U.load_ro(nu, opp, xmnu >> 1);
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    r[i][j] = mkc<R>(0, 0);
#pragma unroll
                    for (int q = 0; q < 3; q++) cmac_cn(r[i][j], t[q][i], v2(q, j));
                }
            add_rows(r);
        }
    }
}

// cm_subgroup with the link and the staple in shared-memory slots and the subgroup (I, J) chosen
// at run time: one copy of the update code serves the three subgroups of a hit.
template <typename R>
__device__ __forceinline__ void cm_subgroup_rt(const StapleSlot<R>& u, const StapleSlot<R>& A, int I, int J,
                                               double c_alpha, const LinkStream& rng, KPDraws& d, bool more,
                                               int* err) {
    Cx<R> ui[3], uj[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        ui[k] = u(I, k);
        uj[k] = u(J, k);
    }
    Cx<R> wii = mkc<R>(0, 0), wij = mkc<R>(0, 0), wji = mkc<R>(0, 0), wjj = mkc<R>(0, 0);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const Cx<R> aki = A(k, I), akj = A(k, J);
        cmac(wii, ui[k], aki);
        cmac(wij, ui[k], akj);
        cmac(wji, uj[k], aki);
        cmac(wjj, uj[k], akj);
    }
    Quat w = {((double)wii.re + (double)wjj.re) / 2.0, ((double)wij.im + (double)wji.im) / 2.0,
              ((double)wij.re - (double)wji.re) / 2.0, ((double)wii.im - (double)wjj.im) / 2.0};
    Quat r = su2_step(c_alpha, w, rng, d, more, err);
    Cx<R> rii = mkc<R>((R)r.a0, (R)r.a3), rjj = mkc<R>((R)r.a0, (R)-r.a3);
    Cx<R> rij = mkc<R>((R)r.a2, (R)r.a1), rji = mkc<R>((R)-r.a2, (R)r.a1);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        Cx<R> ni = rii * ui[k];
        cmac(ni, rij, uj[k]);
        Cx<R> nj = rji * ui[k];
        cmac(nj, rjj, uj[k]);
        u.set(I, k, ni);
        u.set(J, k, nj);
    }
}

// Heatbath update of one link (x, mu) of the (parity, mu) set being swept: no link of the set
// appears in another's staple, so all links of the set update concurrently.  Replaces
// mpi::heatbathcb::hit / sweep (heatbath_mpi.cpp:10-57) for one link; the staple is computed
// once per link, since it does not contain U(x,mu) and is therefore identical for every hit
// (the reference recomputes it per hit).  The staple uses two-row products (staple_rt_rows);
// for FP64 the rebuilt third rows differ from explicit products by the links' distance from
// SU(3) (~1e-15), well inside the 1e-12 parity bound.
//
// With a shared-memory slot (SLOT = true: 18 complexes per thread at slot[k * slot_stride]) the
// staple is accumulated in the slot (staple_rows_into), the link joins it there, and one rolled
// copy of the subgroup update serves all 3 * n_hits updates (cm_subgroup_rt): the hit code is a
// third of the unrolled size and neither phase keeps a 3x3 accumulator in registers (0.217 ms a
// 32^4 FP64 sub-sweep at N_hits = 2 against 0.235 ms with the staple in registers).  Without a
// slot (blocks too large for the static shared memory) the three subgroups are unrolled on
// register-resident matrices.
template <typename R, int NE, int MU, bool SLOT>
__device__ __forceinline__ void hb_link(const Geom& g, const LinkField<R, NE>& U, int par, int h, double c_alpha,
                                        int n_hits, uint64_t seed, uint32_t sweep, int reproject, int* err,
                                        typename V2<R>::T* slot, int slot_stride, uint64_t* link_bar = nullptr) {
    int c[4];
    site_coords(g, par, (uint32_t)h, c);
    const int lex = lex_of(g, c);
    const LinkStream rng(seed, (uint32_t)lex * 4u + (uint32_t)MU, sweep, TAG_HB);  // mod 2^32, as the oracle
    M3<R> u;
    if constexpr (SLOT) {
        const StapleSlot<R> S{slot, slot_stride}, Us{slot + 9 * slot_stride, slot_stride};
        staple_rows_into<R, NE>(g, U, c, lex, par, MU, S);
        KPDraws d = kp_draws_at(rng, 0u);
        if (link_bar) {
            // the block's own links were bulk-copied into the link slots while the staple was formed
            if (!mbar_wait(link_bar, 0u, 1 << 20)) {
                atomicOr(err, (int)DERR_BULK_WAIT);
                return;  // link left unchanged; the host reports the error
            }
        } else {
            Us.put(U.load(MU, par, h));
        }
        const int n_sub = 3 * n_hits;
#pragma unroll 1
        for (int it = 0; it < n_sub; it++) {
            const int sg = it - 3 * (it / 3);  // subgroups (0,1), (1,2), (0,2) in turn
            cm_subgroup_rt<R>(Us, S, sg == 1 ? 1 : 0, sg == 0 ? 1 : 2, c_alpha, rng, d, it + 1 < n_sub, err);
        }
        u = Us.get();
    } else {
        const M3<R> A = staple_rt_rows<R, NE>(g, U, c, lex, par, MU);
        KPDraws d = kp_draws_at(rng, 0u);
        u = U.load(MU, par, h);
        for (int hit = 0; hit < n_hits; hit++) {
            cm_subgroup<R, 0, 1>(u, A, c_alpha, rng, d, true, err);
            cm_subgroup<R, 1, 2>(u, A, c_alpha, rng, d, true, err);
            cm_subgroup<R, 0, 2>(u, A, c_alpha, rng, d, hit + 1 < n_hits, err);
        }
    }
    if (reproject) reproject_fp64(u);
    U.store(MU, par, h, u);
}

// Shared-memory slot of a heatbath block: 18 complexes per thread (staple and link).
template <typename R, int BLOCK>
struct HbSlotFits {
    static constexpr bool value = 18 * BLOCK * sizeof(typename V2<R>::T) <= 48 * 1024;
};

// Single-lattice heatbath launch: one thread per link of the (par, MU) set, geometry as kernel
// parameters.
template <typename R, int NE, int MU>
__global__ void __launch_bounds__(QCB_HB_THREADS, QCB_HB_MINB(R))
    k_hb_subsweep(Geom g, LinkField<R, NE> U, int par, double c_alpha, int n_hits, uint64_t seed, uint32_t sweep,
                  int reproject, int* err) {
    static_assert(HbSlotFits<R, QCB_HB_THREADS>::value, "heatbath slot exceeds static shared memory");
    __shared__ typename V2<R>::T slot[18 * QCB_HB_THREADS];
    uint64_t* link_bar = nullptr;
#if QCB_HB_BULK_LINKS
    // FP64 18-real: the block's own links U_mu(par, h) for its 128 half-sites are 4 whole 32-site
    // tiles, element-major within a tile -- exactly the element-major layout of the link slots --
    // so one thread bulk-copies them there (36 copies of 512 B; tiles past the field are skipped)
    // and the copies land while the staple is formed.
    __shared__ __align__(8) uint64_t bar;
    if constexpr (sizeof(R) == 8 && NE == 9 && QCB_HB_THREADS == 128) {
        if (threadIdx.x == 0) mbar_init(&bar, 1);
        __syncthreads();
        if (threadIdx.x == 0) {
            const int nT = (int)((g.Vh + 31) >> 5);
            const int t0 = blockIdx.x * 4, t1 = min(t0 + 4, nT);
            mbar_expect_tx(&bar, (unsigned)((t1 - t0) * 9 * 32 * sizeof(double2)));
            for (int t = t0; t < t1; t++)
                for (int e = 0; e < 9; e++)
                    bulk_copy_g2s(slot + (9 + e) * 128 + (t - t0) * 32, U.p + U.tile0(MU, par, t * 32) + e * 32,
                                  32 * sizeof(double2), &bar);
        }
        link_bar = &bar;
    }
#endif
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    hb_link<R, NE, MU, true>(g, U, par, (int)h, c_alpha, n_hits, seed, sweep, reproject, err, slot + threadIdx.x,
                             QCB_HB_THREADS, link_bar);
}

// One link's heatbath update (the C ABI's single-link entry, qcb_hb_link; reference
// mpi::heatbathcb::hit, src/heatbath/heatbath_mpi.cpp:10-33).  One thread: the staple A of the
// link, formed with explicit three-row products as compute_staple forms it, goes to a_out
// (9 double2, what hit() leaves in its SU3& argument); then n_hits hits update the link with the
// same arithmetic and the same Philox stream as the (parity, mu) sub-sweep gives that link.
template <typename R, int NE, int MU>
__global__ void k_hb_one(Geom g, LinkField<R, NE> U, int par, int h, double c_alpha, int n_hits, uint64_t seed,
                         uint32_t sweep, int reproject, int* err, double2* a_out) {
    int c[4];
    site_coords(g, par, (uint32_t)h, c);
    const int lex = lex_of(g, c);
    const M3<R> A = staple_rt<R, NE>(g, U, c, lex, par, MU);
#pragma unroll
    for (int k = 0; k < 9; k++) a_out[k] = make_double2((double)A.e[k].re, (double)A.e[k].im);
    hb_link<R, NE, MU, false>(g, U, par, h, c_alpha, n_hits, seed, sweep, reproject, err, nullptr, 0);
}

// ------------------------------------------------------------------ Wilson flow
// One fused RK3 stage (src/flow/gradient_flow.cpp:17-121) for every link (x, mu):
//   F = proj_lie_su3(-U A)                                          compute_force
//   stage 1: Z = F;               W' = exp(eps/4 * F) W             compute_w1
//   stage 2: W' = exp(8/9 eps F - 17/36 eps Z) W;  Z = 8/9 F - 17/36 Z   compute_w2 + replace_force_0
//   stage 3: W' = exp(3/4 eps F - eps Z) W                          compute_w3
// The whole field of forces is never materialised: Win is read-only for the launch and W'
// goes to a second buffer (ping-pong), which is what makes force and update one pass.
template <typename R, int NE, int STAGE, bool MEAS = false>
__device__ __forceinline__ void flow_link(const Geom& g, const LinkField<R, NE>& Win, const LinkField<R, NE>& Wout,
                                          const AlgField<R>& Z, double eps, int mu, int par, int h,
                                          int reproject, const HalfClovers<R>& H = HalfClovers<R>{}) {
    static_assert(!MEAS || (STAGE == 1 && (sizeof(R) == 4 || QCB_FLOW64_ROWS)),
                  "the clover halves come from stage 1's two-row staples");
    int c[4];
    site_coords(g, par, (uint32_t)h, c);
    const int lex = lex_of(g, c);
    M3<R> F, u;
    if constexpr (MEAS) {
        // the same staple and force, with the clover halves of the input configuration
        if constexpr (sizeof(R) == 8) {  // the link reloaded where the halves need it
            const M3<R> A = staple_rt_rows_meas<R, NE>(g, Win, c, lex, par, mu, u, H);
            u = Win.load_ro(mu, par, h);
            F = neg_proj_lie_mul(u, A);
        } else {
            u = Win.load_ro(mu, par, h);
            const M3<R> A = staple_rt_rows_meas<R, NE>(g, Win, c, lex, par, mu, u, H);
            F = neg_proj_lie_mul(u, A);
        }
    } else if constexpr (sizeof(R) == 4 || QCB_FLOW64_ROWS) {
        // two-row staple products and the projection's entries only
        const M3<R> A = staple_rt_rows<R, NE>(g, Win, c, lex, par, mu);
        u = Win.load_ro(mu, par, h);
        F = neg_proj_lie_mul(u, A);
    } else {
        M3<R> A;
#if QCB_FLOW_RTMU
        A = staple_rt<R, NE>(g, Win, c, lex, par, mu);
#else
        switch (mu) {
            case 0: A = staple<R, NE, 0, true>(g, Win, c, lex, par); break;
            case 1: A = staple<R, NE, 1, true>(g, Win, c, lex, par); break;
            case 2: A = staple<R, NE, 2, true>(g, Win, c, lex, par); break;
            default: A = staple<R, NE, 3, true>(g, Win, c, lex, par); break;
        }
#endif
        u = Win.load_ro(mu, par, h);
        F = proj_lie(mul_nn(u, A));
#pragma unroll
        for (int k = 0; k < 9; k++) F.e[k] = mkc<R>(-F.e[k].re, -F.e[k].im);  // proj_lie(-UA) = -proj_lie(UA)
    }
    M3<R> X;
    if (STAGE == 1) {
        const R c1 = (R)(0.25 * eps);
#pragma unroll
        for (int k = 0; k < 9; k++) X.e[k] = scl(c1, F.e[k]);
        Z.store(mu, par, h, F);
    } else if (STAGE == 2) {
        M3<R> z0 = Z.load(mu, par, h);
        const R a = (R)((8.0 / 9.0) * eps), b = (R)((17.0 / 36.0) * eps);
        const R a1 = (R)(8.0 / 9.0), b1 = (R)(17.0 / 36.0);
        M3<R> zn;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            X.e[k] = scl(a, F.e[k]) - scl(b, z0.e[k]);
            zn.e[k] = scl(a1, F.e[k]) - scl(b1, z0.e[k]);
        }
        Z.store(mu, par, h, zn);
    } else {
        M3<R> z0 = Z.load(mu, par, h);
        const R a = (R)(0.75 * eps), b = (R)eps;
#pragma unroll
        for (int k = 0; k < 9; k++) X.e[k] = scl(a, F.e[k]) - scl(b, z0.e[k]);
    }
    M3<R> E = exp_su3(X);
    M3<R> w = mul_nn(E, u);
    // FP32 and 12-real links: one FP64 reprojection per RK3 step, after its last stage (after every
    // stage the FP32 stage took 4-5% longer, with the same flowed Q and E against FP64).
    if (STAGE == 3 && reproject) reproject_fp64(w);
    Wout.store(mu, par, h, w);
}

// Single-lattice RK3 stage.  Grid: blockIdx.x = (site block) * 8 + (mu*2 + parity), so the 8
// link classes of a block of sites run together and share their neighbour links in L2.
template <typename R, int NE, int STAGE>
__global__ void __launch_bounds__(QCB_FLOW1_THREADS, QCB_FLOW1_MINB(R))
    k_flow_stage(Geom g, LinkField<R, NE> Win, LinkField<R, NE> Wout, AlgField<R> Z, double eps, int reproject) {
    const int lt = blockIdx.x & 7;
    const int64_t h = (int64_t)(blockIdx.x >> 3) * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    flow_link<R, NE, STAGE>(g, Win, Wout, Z, eps, lt >> 1, lt & 1, (int)h, reproject);
}

// Stage 1 that also writes the clover halves of its input configuration (the measurement of a
// measured flow step; k_clover_halves completes it).  The links it writes are those of
// k_flow_stage<R, NE, 1>, bit for bit.
template <typename R, int NE>
__global__ void __launch_bounds__(QCB_FLOW1_THREADS, QCB_FLOW_MEAS_MINB(R))
    k_flow_stage1_meas(Geom g, LinkField<R, NE> Win, LinkField<R, NE> Wout, AlgField<R> Z, double eps, int reproject,
                       HalfClovers<R> H) {
    const int lt = blockIdx.x & 7;
    const int64_t h = (int64_t)(blockIdx.x >> 3) * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    flow_link<R, NE, 1, true>(g, Win, Wout, Z, eps, lt >> 1, lt & 1, (int)h, reproject, H);
}

// ------------------------------------------------------------------ the reference's separate flow passes
// GradientFlow's member passes (src/flow/gradient_flow.cpp:17-121), for callers that drive them one
// by one; rk3_step runs the fused stages above.  Forces are su(3) fields in the accumulator layout.
// compute_force: F = proj_lie_su3(-U A) of every link, with the fused stage's staple and projection.
// Grid: blockIdx.x = (site block) * 8 + (mu*2 + parity), as the fused stage.
template <typename R, int NE>
__global__ void __launch_bounds__(QCB_FLOW1_THREADS) k_flow_force(Geom g, LinkField<R, NE> W, AlgField<R> F) {
    const int lt = blockIdx.x & 7;
    const int64_t h = (int64_t)(blockIdx.x >> 3) * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    const int mu = lt >> 1, par = lt & 1;
    int c[4];
    site_coords(g, par, (uint32_t)h, c);
    const int lex = lex_of(g, c);
    const M3<R> A = staple_rt_rows<R, NE>(g, W, c, lex, par, mu);
    const M3<R> u = W.load_ro(mu, par, (int)h);
    F.store(mu, par, (int)h, neg_proj_lie_mul(u, A));
}

// compute_w1 / w2 / w3: W <- exp(X) W in place (a link's update reads only that link and its
// forces), X = c F0 (use_f1 = 0, c = a) or a F1 - b F0; FP32 and 12-real links reprojected after
// compute_w3 (the caller passes reproject = 0 for w1 and w2), as after the fused third stage.
template <typename R, int NE>
__global__ void __launch_bounds__(256) k_flow_update(Geom g, LinkField<R, NE> W, AlgField<R> F0, AlgField<R> F1,
                                                     double a, double b, int use_f1, int reproject) {
    const int lt = blockIdx.y, mu = lt >> 1, par = lt & 1;
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    const M3<R> z0 = F0.load(mu, par, (int)h);
    M3<R> X;
    if (use_f1) {
        const M3<R> z1 = F1.load(mu, par, (int)h);
#pragma unroll
        for (int k = 0; k < 9; k++) X.e[k] = scl((R)a, z1.e[k]) - scl((R)b, z0.e[k]);
    } else {
#pragma unroll
        for (int k = 0; k < 9; k++) X.e[k] = scl((R)a, z0.e[k]);
    }
    M3<R> w = mul_nn(exp_su3(X), W.load(mu, par, (int)h));
    if (reproject) reproject_fp64(w);
    W.store(mu, par, (int)h, w);
}

// replace_force_0: F0 <- 8/9 F1 - 17/36 F0.
template <typename R>
__global__ void __launch_bounds__(256) k_flow_replace(int64_t Vh, AlgField<R> F0, AlgField<R> F1) {
    const int lt = blockIdx.y, mu = lt >> 1, par = lt & 1;
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= Vh) return;
    const M3<R> z0 = F0.load(mu, par, (int)h), z1 = F1.load(mu, par, (int)h);
    const R a1 = (R)(8.0 / 9.0), b1 = (R)(17.0 / 36.0);
    M3<R> zn;
#pragma unroll
    for (int k = 0; k < 9; k++) zn.e[k] = scl(a1, z1.e[k]) - scl(b1, z0.e[k]);
    F0.store(mu, par, (int)h, zn);
}

// ------------------------------------------------------------------ reductions
// Block reduction of NV doubles -> partials[blockIdx * NV + k] (warp shuffles, then one
// warp).  Component k is a maximum when bit k of MAXMASK is set, a sum otherwise.
template <int NV, unsigned MAXMASK = 0u>
__device__ __forceinline__ void block_sum_store(double v[NV], double* partials, int block_id) {
    __shared__ double sm[32][NV];
#pragma unroll
    for (int k = 0; k < NV; k++)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            double o = __shfl_down_sync(0xffffffffu, v[k], off);
            v[k] = ((MAXMASK >> k) & 1u) ? fmax(v[k], o) : v[k] + o;
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) sm[wid][k] = v[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double s = lane < nw ? sm[lane][k] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                double o = __shfl_down_sync(0xffffffffu, s, off);
                s = ((MAXMASK >> k) & 1u) ? fmax(s, o) : s + o;
            }
            if (lane == 0) partials[(size_t)block_id * NV + k] = s;
        }
    }
}

// Deterministic final sum of nb partial vectors (one block of 256 threads; fixed order).
// mode bit k set: component k is a max instead of a sum.
__global__ void k_finalize(const double* partials, int nb, int nv, unsigned max_mask, double* out);

// Plaquette (observables_mpi.cpp:11-35): per site sum over mu<nu of Re Tr(U_mu(x) U_nu(x+mu)
// U_mu(x+nu)^dag U_nu(x)^dag)/3, evaluated as Re Tr((U_mu(x) U_nu(x+mu)) (U_nu(x) U_mu(x+nu))^dag).
// Plaquette sum of one site: sum over mu<nu of Re Tr(U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag)/3
// (observables_mpi.cpp:11-35), evaluated as Re Tr((U_mu(x) U_nu(x+mu)) (U_nu(x) U_mu(x+nu))^dag).
template <typename R, int NE, bool TILED>
__device__ __forceinline__ double site_plaquette(const Geom& g, const LinkField<R, NE, TILED>& U, int par, int h) {
    int c[4];
    site_coords(g, par, (uint32_t)h, c);
    const int lex = lex_of(g, c);
    double s = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; mu++) {
        const int xmu = step_up(g, lex, c[mu], mu);
        M3<R> umu = U.load_ro(mu, par, h);
#pragma unroll
        for (int nu = mu + 1; nu < 4; nu++) {
            const int xnu = step_up(g, lex, c[nu], nu);
            M3<R> p1 = mul_nn(umu, U.load_ro(nu, par ^ 1, xmu >> 1));
            M3<R> p2 = mul_nn(U.load_ro(nu, par, h), U.load_ro(mu, par ^ 1, xnu >> 1));
            s += (double)re_tr_mul_na(p1, p2) / 3.0;
        }
    }
    return s;
}

// Grid (2, site blocks): the parity is the fast grid dimension, so the two blocks of one site range
// run together and share their neighbour links in L2 (with the parity as the slow dimension each
// parity streamed the whole field: 2.1x the algorithmic DRAM bytes at 32^4 FP64).
template <typename R, int NE, bool TILED = true>
__global__ void __launch_bounds__(256) k_plaquette(Geom g, LinkField<R, NE, TILED> U, double* partials) {
    const int par = blockIdx.x;
    double v[1] = {0.0};
    for (int64_t h = (int64_t)blockIdx.y * blockDim.x + threadIdx.x; h < g.Vh; h += (int64_t)gridDim.y * blockDim.x)
        v[0] += site_plaquette(g, U, par, (int)h);
    block_sum_store<1>(v, partials, blockIdx.y * gridDim.x + blockIdx.x);
}

// Clover field strength F = (C - C^dag)/8 (clover_site, observables_mpi.cpp:66-90) held as its
// nine independent reals: F is exactly anti-Hermitian, so only the upper off-diagonal entries
// o = (F01, F02, F12) and the imaginary diagonal d_i = Im F_ii are kept.
template <typename R>
struct CloverF {
    Cx<R> o[3];
    R d[3];
};

// Adds leaf L to the clover sums: o_ij += L_ij - conj(L_ji) (i < j), d_i += Im L_ii.
template <typename R>
__device__ __forceinline__ void clover_acc(CloverF<R>& S, const M3<R>& L) {
    S.o[0] = S.o[0] + (L(0, 1) - cconj(L(1, 0)));
    S.o[1] = S.o[1] + (L(0, 2) - cconj(L(2, 0)));
    S.o[2] = S.o[2] + (L(1, 2) - cconj(L(2, 1)));
#pragma unroll
    for (int i = 0; i < 3; i++) S.d[i] += L(i, i).im;
}

// Row i of a link or of its adjoint.
template <typename R, bool DAG>
__device__ __forceinline__ void link_row(const M3<R>& A, int i, Cx<R> r[3]) {
#pragma unroll
    for (int k = 0; k < 3; k++) r[k] = DAG ? cconj(A(k, i)) : A(i, k);
}
// r <- r B (DAG = false) or r B^dag (DAG = true) for the two rows r[0], r[1].
template <typename R, bool DAG>
__device__ __forceinline__ void rows_mul(Cx<R> r[2][3], const M3<R>& B) {
#pragma unroll
    for (int i = 0; i < 2; i++) {
        Cx<R> n[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            n[j] = mkc<R>(0, 0);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                if (DAG)
                    cmac_nc(n[j], r[i][k], B(j, k));
                else
                    cmac(n[j], r[i][k], B(k, j));
            }
        }
#pragma unroll
        for (int j = 0; j < 3; j++) r[i][j] = n[j];
    }
}
// Full SU(3) matrix from its first two rows: r2 = conj(r0 x r1).
template <typename R>
__device__ __forceinline__ M3<R> from_rows(const Cx<R> r[2][3]) {
    M3<R> L;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        L(0, j) = r[0][j];
        L(1, j) = r[1][j];
        const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        L(2, j) = cconj(r[0][j1] * r[1][j2] - r[0][j2] * r[1][j1]);
    }
    return L;
}

// One clover leaf A' B' C' D' (' = adjoint where the flag is set), in the reference's association
// ((A' B') C') D'.  The first two rows are carried through the three products and the third row
// of the SU(3) leaf is rebuilt (60 instead of 81 complex multiply-adds; the rebuilt row differs
// from the product by the links' distance from SU(3): ~1e-15 in FP64, the FP32 rounding level in
// FP32).  With QCB_CLOVER64_ROWS = 0, FP64 multiplies full matrices.
template <typename R, bool DA, bool DB, bool DC, bool DD>
__device__ __forceinline__ M3<R> clover_leaf(const M3<R>& A, const M3<R>& B, const M3<R>& C, const M3<R>& D) {
    if constexpr (sizeof(R) == 4 || QCB_CLOVER64_ROWS) {
        Cx<R> r[2][3];
        link_row<R, DA>(A, 0, r[0]);
        link_row<R, DA>(A, 1, r[1]);
        rows_mul<R, DB>(r, B);
        rows_mul<R, DC>(r, C);
        rows_mul<R, DD>(r, D);
        return from_rows(r);
    } else {
        const M3<R> a = DA ? adjoint(A) : A;
        M3<R> t = DB ? mul_na(a, B) : mul_nn(a, B);
        t = DC ? mul_na(t, C) : mul_nn(t, C);
        return DD ? mul_na(t, D) : mul_nn(t, D);
    }
}

// F of plane (mu, nu) at site x with the four leaves in the reference's order; also returns
// Re Tr of leaf 1, which is the plaquette U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag.
template <typename R, int NE>
__device__ __forceinline__ CloverF<R> clover_F(const LinkField<R, NE>& U, const Steps& st, int lex, int par, int mu,
                                               int nu, R& plaq_tr) {
    const int opp = par ^ 1;
    const int upnu = sel4(st.up, nu), dnnu = sel4(st.dn, nu);
    const int xpmu = lex + sel4(st.up, mu), xpnu = lex + upnu;
    const int xmmu = lex + sel4(st.dn, mu), xmnu = lex + dnnu;
    // x+-mu have the nu coordinate of x
    const int xmmupnu = xmmu + upnu, xmmumnu = xmmu + dnnu;
    const int xpmumnu = xpmu + dnnu;
    const int h = lex >> 1;
    CloverF<R> S;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        S.o[k] = mkc<R>(0, 0);
        S.d[k] = R(0);
    }
    M3<R> L;
    // leaf 1: U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
    L = clover_leaf<R, false, false, true, true>(U.load_ro(mu, par, h), U.load_ro(nu, opp, xpmu >> 1),
                                                 U.load_ro(mu, opp, xpnu >> 1), U.load_ro(nu, par, h));
    plaq_tr = (L(0, 0).re + L(1, 1).re) + L(2, 2).re;
    clover_acc(S, L);
    // leaf 2: U_nu(x) U_mu(x-mu+nu)^dag U_nu(x-mu)^dag U_mu(x-mu)
    L = clover_leaf<R, false, true, true, false>(U.load_ro(nu, par, h), U.load_ro(mu, par, xmmupnu >> 1),
                                                 U.load_ro(nu, opp, xmmu >> 1), U.load_ro(mu, opp, xmmu >> 1));
    clover_acc(S, L);
    // leaf 3: U_mu(x-mu)^dag U_nu(x-mu-nu)^dag U_mu(x-mu-nu) U_nu(x-nu)
    L = clover_leaf<R, true, true, false, false>(U.load_ro(mu, opp, xmmu >> 1), U.load_ro(nu, par, xmmumnu >> 1),
                                                 U.load_ro(mu, par, xmmumnu >> 1), U.load_ro(nu, opp, xmnu >> 1));
    clover_acc(S, L);
    // leaf 4: U_nu(x-nu)^dag U_mu(x-nu) U_nu(x+mu-nu) U_mu(x)^dag
    L = clover_leaf<R, true, false, false, true>(U.load_ro(nu, opp, xmnu >> 1), U.load_ro(mu, opp, xmnu >> 1),
                                                 U.load_ro(nu, par, xpmumnu >> 1), U.load_ro(mu, par, h));
    clover_acc(S, L);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        S.o[k] = scl((R)0.125, S.o[k]);
        S.d[k] = (R)0.25 * S.d[k];  // Im F_ii = (Im C_ii - (-Im C_ii)) / 8
    }
    return S;
}

// Re Tr(Fa Fb) and |F|^2 of anti-Hermitian matrices from their nine reals:
//   Re Tr(Fa Fb) = -2 sum_k Re(oa_k conj(ob_k)) - sum_i da_i db_i,  |F|^2 = 2 sum_k |o_k|^2 + sum_i d_i^2.
// FP32 clover pass: the per-site traces Re Tr(Fa Fb) and |F|^2 in FP32 (the global sums of q, e
// and the plaquette stay FP64): 0.341 against 0.348 ms at 32^4, with the site values' FP32 rounding
// (~1e-7 relative) far inside the |dQ| < 1e-4 and dE/E < 1e-6 bounds of the FP32 forms.
#ifndef QCB_CLOVER32_SITE
#define QCB_CLOVER32_SITE 1
#endif
template <typename R>
__device__ __forceinline__ double clover_re_tr(const CloverF<R>& a, const CloverF<R>& b) {
    if constexpr (sizeof(R) == 4 && QCB_CLOVER32_SITE) {
        float s = 0.f, t = 0.f;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            s = fmaf(a.o[k].re, b.o[k].re, fmaf(a.o[k].im, b.o[k].im, s));
            t = fmaf(a.d[k], b.d[k], t);
        }
        return (double)(-2.f * s - t);
    }
    double s = 0.0, t = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        s += (double)a.o[k].re * (double)b.o[k].re + (double)a.o[k].im * (double)b.o[k].im;
        t += (double)a.d[k] * (double)b.d[k];
    }
    return -2.0 * s - t;
}
template <typename R>
__device__ __forceinline__ double clover_sq_norm(const CloverF<R>& a) {
    if constexpr (sizeof(R) == 4 && QCB_CLOVER32_SITE) {
        float s = 0.f, t = 0.f;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            s = fmaf(a.o[k].re, a.o[k].re, fmaf(a.o[k].im, a.o[k].im, s));
            t = fmaf(a.d[k], a.d[k], t);
        }
        return (double)(2.f * s + t);
    }
    double s = 0.0, t = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        s += (double)a.o[k].re * (double)a.o[k].re + (double)a.o[k].im * (double)a.o[k].im;
        t += (double)a.d[k] * (double)a.d[k];
    }
    return 2.0 * s + t;
}

// local_q_e_clover (observables_mpi.cpp:93-112) for one (site, plane pair):
// pair 0: +Re Tr(F01 F23), pair 1: -Re Tr(F02 F13), pair 2: +Re Tr(F03 F12); e += |F|^2/2.
// Adds (q/(4 pi^2), e) to v[0], v[1] and, with NV = 3, the plaquette sum Re Tr(leaf 1)/3 of the
// pair's two planes to v[2] (the three pairs cover the six planes once).
template <typename R, int NE, int NV>
__device__ __forceinline__ void site_clover_pair(const Geom& g, const LinkField<R, NE>& U, int par, int pair, int h,
                                                 double v[NV]) {
    const int a_mu = 0, a_nu = pair + 1;
    const int b_mu = (pair == 0) ? 2 : 1, b_nu = (pair == 2) ? 2 : 3;
    int c[4];
    site_coords(g, par, (uint32_t)h, c);
    const int lex = lex_of(g, c);
    const Steps st = make_steps(g, c);
    R pa, pb;
    CloverF<R> Fa, Fb;
    if constexpr (NE == 6) {
        // 12-real links: one rolled copy of the clover code serves both planes.  With the third rows
        // rebuilt for every loaded link, two unrolled clovers overflow the instruction cache: 32^4
        // clover pass 0.695 against 0.734 ms FP64-12, 0.391 against 0.411 ms FP32-12, bit-identical
        // (for 18-real links the rolled loop is slower: 0.674 against 0.623 ms FP64, 0.374 against
        // 0.344-0.354 ms FP32).
#pragma unroll 1
        for (int k = 0; k < 2; k++) {
            R p;
            const CloverF<R> F = clover_F(U, st, lex, par, k ? b_mu : a_mu, k ? b_nu : a_nu, p);
            if (k == 0) {
                Fa = F;
                pa = p;
            } else {
                Fb = F;
                pb = p;
            }
        }
    } else {
        Fa = clover_F(U, st, lex, par, a_mu, a_nu, pa);
        Fb = clover_F(U, st, lex, par, b_mu, b_nu, pb);
    }
    const double q = clover_re_tr(Fa, Fb);
    v[0] += (pair == 1 ? -q : q) * (1.0 / (4.0 * kPi * kPi));
    v[1] += 0.5 * (clover_sq_norm(Fa) + clover_sq_norm(Fb));
    if constexpr (NV == 3) v[2] += ((double)pa + (double)pb) / 3.0;
}

// Clover Q/E of one field: grid (6 = parity x plane pair, site blocks); partials (q, e, p) per
// block, p the plaquette sum of the block's planes.  The (parity, pair) class is the fast grid
// dimension, so the six blocks of one site range run together and share their links in L2 (with
// the class as the slow dimension every class streamed the whole field: 7-9x the algorithmic DRAM
// bytes at 32^4).
template <typename R, int NE>
__global__ void __launch_bounds__(128, QCB_CLOVER_MINB(R)) k_clover_qe(Geom g, LinkField<R, NE> U, double* partials) {
    const int par = blockIdx.x & 1, pair = blockIdx.x >> 1;
    double v[3] = {0.0, 0.0, 0.0};
    for (int64_t h = (int64_t)blockIdx.y * blockDim.x + threadIdx.x; h < g.Vh; h += (int64_t)gridDim.y * blockDim.x)
        site_clover_pair<R, NE, 3>(g, U, par, pair, (int)h, v);
    block_sum_store<3>(v, partials, blockIdx.y * gridDim.x + blockIdx.x);
}

// The measurement from the clover halves: per site, F of each plane = (half 0 + half 1) scaled as
// clover_F scales its leaf sums, then q, e and the plaquette sum as site_clover_pair forms them.
// One thread per site (site = parity * Vh + h), partials (q, e, p) per block.
template <typename R>
__device__ __forceinline__ void site_halves_qe(const HalfClovers<R>& H, int64_t site, double v[3]) {
    {
        CloverF<R> F[6];
        double pl = 0.0;
#pragma unroll
        for (int p = 0; p < 6; p++) {
            R x[9];
#pragma unroll
            for (int k = 0; k < 9; k++) x[k] = H.half(p, 0, k, site) + H.half(p, 1, k, site);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                F[p].o[k] = scl((R)0.125, mkc<R>(x[2 * k], x[2 * k + 1]));
                F[p].d[k] = (R)0.25 * x[6 + k];
            }
            pl += (double)H.plaq(p, site);
        }
        // pairs 01-23 (+), 02-13 (-), 03-12 (+)
        const double q = clover_re_tr(F[0], F[5]) - clover_re_tr(F[1], F[4]) + clover_re_tr(F[2], F[3]);
        v[0] = q * (1.0 / (4.0 * kPi * kPi));
        double e = 0.0;
#pragma unroll
        for (int p = 0; p < 6; p++) e += clover_sq_norm(F[p]);
        v[1] = 0.5 * e;
        v[2] = pl / 3.0;
    }
}
template <typename R>
__global__ void __launch_bounds__(128) k_clover_halves(Geom g, HalfClovers<R> H, double* partials) {
    double v[3] = {0.0, 0.0, 0.0};
    const int64_t site = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (site < H.V) site_halves_qe(H, site, v);
    block_sum_store<3>(v, partials, blockIdx.x);
}

// clover_site (observables_mpi.cpp:66-90) at one site, plane (mu, nu), as the 3x3 F (18 doubles), or
// with mu < 0 local_q_e_clover (:93-112): out[0] = q/(4 pi^2) summed over the three plane pairs,
// out[1] = e.  One thread.
template <typename R, int NE>
__global__ void k_clover_site(Geom g, LinkField<R, NE> U, int par, int h, int mu, int nu, double* out) {
    if (mu >= 0) {
        int c[4];
        site_coords(g, par, (uint32_t)h, c);
        const int lex = lex_of(g, c);
        const Steps st = make_steps(g, c);
        R p;
        const CloverF<R> F = clover_F(U, st, lex, par, mu, nu, p);
        const Cx<R> o[3][3] = {{mkc<R>(0, F.d[0]), F.o[0], F.o[1]},
                               {mkc<R>(-F.o[0].re, F.o[0].im), mkc<R>(0, F.d[1]), F.o[2]},
                               {mkc<R>(-F.o[1].re, F.o[1].im), mkc<R>(-F.o[2].re, F.o[2].im), mkc<R>(0, F.d[2])}};
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                out[2 * (3 * i + j)] = (double)o[i][j].re;
                out[2 * (3 * i + j) + 1] = (double)o[i][j].im;
            }
    } else {
        double v[2] = {0.0, 0.0};
        for (int pair = 0; pair < 3; pair++) site_clover_pair<R, NE, 2>(g, U, par, pair, h, v);
        out[0] = v[0];
        out[1] = v[1];
    }
}

// Unitarity error ||U U^dag - 1||_F per link (src/bin/test.cpp:58-72): partials (max, sum).
template <typename R, int NE>
__global__ void __launch_bounds__(256) k_unitarity(Geom g, LinkField<R, NE> U, double* partials) {
    const int lt = blockIdx.y;
    const int mu = lt >> 1, par = lt & 1;
    double v[2] = {0.0, 0.0};
    for (int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; h < g.Vh; h += (int64_t)gridDim.x * blockDim.x) {
        M3<double> u = convert<double>(U.load_ro(mu, par, (int)h));
        M3<double> d = mul_na(u, u);
        d(0, 0).re -= 1.0;
        d(1, 1).re -= 1.0;
        d(2, 2).re -= 1.0;
        double err = sqrt(sq_norm(d));
        v[0] = fmax(v[0], err);
        v[1] += err;
    }
    block_sum_store<2, 1u>(v, partials, blockIdx.y * gridDim.x + blockIdx.x);
}

// ------------------------------------------------------------------ layout, starts, shift
// AoS (site lex, mu, row-major 3x3 complex; optionally big-endian) -> parity-split SoA.
template <typename R, int NE>
__global__ void k_aos_to_soa(Geom g, const double2* aos, LinkField<R, NE> U, int bswap) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.V * 4) return;
    const int lex = (int)(t >> 2);
    const int mu = (int)(t & 3);
    int c[4];
    lex_coords(g, lex, c);
    const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    M3<R> u;
#pragma unroll
    for (int e = 0; e < 9; e++) {
        double2 v = aos[t * 9 + e];
        if (bswap) {
            v.x = bswap_f64(v.x);
            v.y = bswap_f64(v.y);
        }
        u.e[e] = mkc<R>((R)v.x, (R)v.y);
    }
    U.store(mu, par, lex >> 1, u);
}
template <typename R, int NE>
__global__ void k_soa_to_aos(Geom g, LinkField<R, NE> U, double2* aos, int bswap) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.V * 4) return;
    const int lex = (int)(t >> 2);
    const int mu = (int)(t & 3);
    int c[4];
    lex_coords(g, lex, c);
    const int par = (c[0] + c[1] + c[2] + c[3]) & 1;
    M3<R> u = U.load_ro(mu, par, lex >> 1);
#pragma unroll
    for (int e = 0; e < 9; e++) {
        double2 v;
        v.x = (double)u.e[e].re;
        v.y = (double)u.e[e].im;
        if (bswap) {
            v.x = bswap_f64(v.x);
            v.y = bswap_f64(v.y);
        }
        aos[t * 9 + e] = v;
    }
}

// cold_start (GaugeField.cpp:23-33) / hot_start (GaugeField.cpp:10-20) with a Haar SU(3)
// generator: two complex Gaussian columns from the link's Philox stream (Box-Muller),
// orthonormalised and completed by projection_su3 (GaugeField.cpp:36-58), in double.
template <typename R, int NE>
__global__ void k_start(Geom g, LinkField<R, NE> U, int hot, uint64_t seed) {
    const int lt = blockIdx.y;
    const int mu = lt >> 1, par = lt & 1;
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    M3<double> m;
    if (!hot) {
        m = ident<double>();
    } else {
        int c[4];
        site_coords(g, par, (uint32_t)h, c);
        const int lex = lex_of(g, c);
        LinkStream rng(seed, (uint32_t)lex * 4u + (uint32_t)mu, 0u, TAG_HOT);
        double gs[12];
#pragma unroll
        for (int k = 0; k < 12; k += 2) {
            double u1 = rng.next(), u2 = rng.next();
            double r = sqrt(-2.0 * log(1.0 - u1));
            double s, co;
            sincospi(2.0 * u2, &s, &co);
            gs[k] = r * co;
            gs[k + 1] = r * s;
        }
        set_zero(m);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            m(i, 0) = mkc(gs[2 * i], gs[2 * i + 1]);
            m(i, 1) = mkc(gs[6 + 2 * i], gs[6 + 2 * i + 1]);
        }
        project_su3(m);
    }
    U.store(mu, par, (int)h, convert<R>(m));
}

// U'(x) = U(x - s) (the global translation of Shift.cpp:109-160 on one periodic lattice).
template <typename R, int NE>
__global__ void k_shift(Geom g, LinkField<R, NE> src, LinkField<R, NE> dst, int s0, int s1, int s2, int s3) {
    const int lt = blockIdx.y;
    const int mu = lt >> 1, par = lt & 1;
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    int c[4];
    site_coords(g, par, (uint32_t)h, c);
    const int s[4] = {s0, s1, s2, s3};
#pragma unroll
    for (int d = 0; d < 4; d++) {
        int v = c[d] - s[d];
        if (v < 0) v += g.L[d];
        c[d] = v;
    }
    const int spar = (c[0] + c[1] + c[2] + c[3]) & 1;
    const int slex = lex_of(g, c);
    dst.copy_from(mu, par, (int)h, src, spar, slex >> 1);
}

// projection_su3 of every link, in double (GaugeField.cpp:61-71).
template <typename R, int NE>
__global__ void k_reunitarize(Geom g, LinkField<R, NE> U) {
    const int lt = blockIdx.y;
    const int mu = lt >> 1, par = lt & 1;
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    M3<double> u = convert<double>(U.load(mu, par, (int)h));
    project_su3(u);
    U.store(mu, par, (int)h, convert<R>(u));
}

// Staple field of one direction, written in AoS order (diagnostic entry point).
// Loads one link (mu, par, h) and stores its trace: the probe through which a test shows the
// checked build catching an index outside the field.
template <typename R, int NE>
__global__ void k_probe_link(LinkField<R, NE> U, int mu, int par, int h, double* out) {
    const M3<R> u = U.load(mu, par, h);
    out[0] = (double)(u(0, 0).re + u(1, 1).re + u(2, 2).re);
}

template <typename R, int NE, int MU>
__global__ void k_staple_field(Geom g, LinkField<R, NE> U, double2* out) {
    const int par = blockIdx.y;
    const int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= g.Vh) return;
    int c[4];
    site_coords(g, par, (uint32_t)h, c);
    const int lex = lex_of(g, c);
    M3<R> A = staple<R, NE, MU, true>(g, U, c, lex, par);
#pragma unroll
    for (int e = 0; e < 9; e++) {
        double2 v;
        v.x = (double)A.e[e].re;
        v.y = (double)A.e[e].im;
        out[(int64_t)lex * 9 + e] = v;
    }
}

}  // namespace qcb
