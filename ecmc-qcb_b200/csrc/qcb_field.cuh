// qcb_field.cuh -- lattice geometry, parity-split SoA link storage and the Philox link streams.
//
// Geometry follows the reference's GeometryCB conventions (src/geometry/GeometryCB.h:25-27,
// GeometryCB.cpp:57-67): lexicographic site index with x fastest and t slowest, direction
// order mu = x,y,z,t, site parity (x+y+z+t) mod 2.  The reference's (L+2)^4 halo box, its
// neighbour table and frozen-link mask are replaced by periodic coordinate arithmetic on a
// single periodic lattice: one GPU holds the whole lattice, so there is no halo to refresh.
//
// HBM layout of one field ("parity-split structure of arrays"):
//     plane(mu, parity, e) = (mu*2 + parity)*NE + e,        e = 3*row + col
//     element = base[ plane * Vh + h ]                       (one complex per element)
// where h = lex/2 is the half-site index inside its parity (Lx is even, so the two sites
// 2k, 2k+1 of an x-row have opposite parity and share h = k).  Consecutive threads own
// consecutive h, so every element load is a fully coalesced 16-byte (FP64) or 8-byte
// (FP32) access.  NE = 9 stores the full matrix (18 reals); NE = 6 stores the first two
// rows (12 reals) and rebuilds the third in registers as conj(row0 x row1).
#pragma once
#include <stdint.h>

#include "qcb_su3.cuh"

namespace qcb {

template <typename R>
struct V2;
template <>
struct V2<double> {
    using T = double2;
};
template <>
struct V2<float> {
    using T = float2;
};

struct Geom {
    int L[4];
    int stride[4];  // lexicographic strides (1, Lx, Lx*Ly, Lx*Ly*Lz)
    int64_t V, Vh;
};

inline Geom make_geom(const int L[4]) {
    Geom g;
    for (int d = 0; d < 4; d++) g.L[d] = L[d];
    g.stride[0] = 1;
    g.stride[1] = L[0];
    g.stride[2] = L[0] * L[1];
    g.stride[3] = L[0] * L[1] * L[2];
    g.V = (int64_t)L[0] * L[1] * L[2] * L[3];
    g.Vh = g.V / 2;
    return g;
}

// Coordinates of half-site h of the given parity.
QCB_HD void site_coords(const Geom& g, int par, uint32_t h, int c[4]) {
    uint32_t i = 2u * h;
    uint32_t L0 = g.L[0], L1 = g.L[1], L2 = g.L[2];
    c[0] = (int)(i % L0);
    i /= L0;
    c[1] = (int)(i % L1);
    i /= L1;
    c[2] = (int)(i % L2);
    c[3] = (int)(i / L2);
    c[0] += (c[1] + c[2] + c[3] + par) & 1;
}
QCB_HD int64_t lex_of(const Geom& g, const int c[4]) {
    return (int64_t)c[0] + (int64_t)c[1] * g.stride[1] + (int64_t)c[2] * g.stride[2] + (int64_t)c[3] * g.stride[3];
}
QCB_HD void lex_coords(const Geom& g, int64_t lex, int c[4]) {
    c[0] = (int)(lex % g.L[0]);
    lex /= g.L[0];
    c[1] = (int)(lex % g.L[1]);
    lex /= g.L[1];
    c[2] = (int)(lex % g.L[2]);
    c[3] = (int)(lex / g.L[2]);
}
// lex index of the site one step up / down in direction d from a site with coordinate cd.
QCB_HD int64_t step_up(const Geom& g, int64_t lex, int cd, int d) {
    return (cd == g.L[d] - 1) ? lex - (int64_t)(g.L[d] - 1) * g.stride[d] : lex + g.stride[d];
}
QCB_HD int64_t step_dn(const Geom& g, int64_t lex, int cd, int d) {
    return (cd == 0) ? lex + (int64_t)(g.L[d] - 1) * g.stride[d] : lex - g.stride[d];
}

// Link storage view; NE = 9 (18 reals) or 6 (12 reals, third row rebuilt on load).
template <typename R, int NE>
struct LinkField {
    typedef typename V2<R>::T C2;
    C2* p;
    int64_t Vh;
    QCB_HD size_t plane(int mu, int par, int e) const { return (size_t)((mu * 2 + par) * NE + e) * (size_t)Vh; }
    __device__ __forceinline__ M3<R> load(int mu, int par, int64_t h) const {
        M3<R> u;
        const C2* b = p + plane(mu, par, 0) + h;
#pragma unroll
        for (int e = 0; e < NE; e++) {
            C2 v = b[(size_t)e * Vh];
            u.e[e] = mkc<R>(v.x, v.y);
        }
        if (NE == 6) rebuild_row2(u);
        return u;
    }
    // read-only path for links that no thread of the running kernel writes
    __device__ __forceinline__ M3<R> load_ro(int mu, int par, int64_t h) const {
        M3<R> u;
        const C2* b = p + plane(mu, par, 0) + h;
#pragma unroll
        for (int e = 0; e < NE; e++) {
            C2 v = __ldg(b + (size_t)e * Vh);
            u.e[e] = mkc<R>(v.x, v.y);
        }
        if (NE == 6) rebuild_row2(u);
        return u;
    }
    __device__ __forceinline__ void store(int mu, int par, int64_t h, const M3<R>& u) const {
        C2* b = p + plane(mu, par, 0) + h;
#pragma unroll
        for (int e = 0; e < NE; e++) {
            C2 v;
            v.x = u.e[e].re;
            v.y = u.e[e].im;
            b[(size_t)e * Vh] = v;
        }
    }
};

// su(3) algebra storage: 8 reals per link as 4 complex planes
//   0: Z01, 1: Z02, 2: Z12, 3: (Im Z00, Im Z11);  Z22 = -i(Im Z00 + Im Z11), Zji = -conj(Zij).
template <typename R>
struct AlgField {
    typedef typename V2<R>::T C2;
    C2* p;
    int64_t Vh;
    QCB_HD size_t plane(int mu, int par, int e) const { return (size_t)((mu * 2 + par) * 4 + e) * (size_t)Vh; }
    __device__ __forceinline__ M3<R> load(int mu, int par, int64_t h) const {
        const C2* b = p + plane(mu, par, 0) + h;
        C2 z01 = b[0], z02 = b[(size_t)Vh], z12 = b[2 * (size_t)Vh], dg = b[3 * (size_t)Vh];
        M3<R> z;
        z(0, 1) = mkc<R>(z01.x, z01.y);
        z(0, 2) = mkc<R>(z02.x, z02.y);
        z(1, 2) = mkc<R>(z12.x, z12.y);
        z(1, 0) = mkc<R>(-z01.x, z01.y);
        z(2, 0) = mkc<R>(-z02.x, z02.y);
        z(2, 1) = mkc<R>(-z12.x, z12.y);
        z(0, 0) = mkc<R>(0, dg.x);
        z(1, 1) = mkc<R>(0, dg.y);
        z(2, 2) = mkc<R>(0, -(dg.x + dg.y));
        return z;
    }
    __device__ __forceinline__ void store(int mu, int par, int64_t h, const M3<R>& z) const {
        C2* b = p + plane(mu, par, 0) + h;
        C2 v;
        v.x = z(0, 1).re;
        v.y = z(0, 1).im;
        b[0] = v;
        v.x = z(0, 2).re;
        v.y = z(0, 2).im;
        b[(size_t)Vh] = v;
        v.x = z(1, 2).re;
        v.y = z(1, 2).im;
        b[2 * (size_t)Vh] = v;
        v.x = z(0, 0).im;
        v.y = z(1, 1).im;
        b[3 * (size_t)Vh] = v;
    }
};

// ------------------------------------------------------------------ Philox4x32-10
// Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3" (SC'11).
QCB_HD void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
        uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
#else
        uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

// Stream tags (counter word 3).
enum : uint32_t { TAG_HB = 0x48420001u, TAG_HOT = 0x484F5401u, TAG_SHIFT = 0x53480001u };

QCB_HD double u53(uint32_t hi, uint32_t lo) {
    uint64_t v = ((uint64_t)hi << 32) | lo;
    return (double)(v >> 11) * 0x1.0p-53;
}

// Per-link uniform stream keyed on (seed) and countered on (draw, link, sweep, tag): the
// numbers a link receives do not depend on launch shape, block size or thread count.
struct LinkStream {
    uint32_t k0, k1, link, sweep, tag, n;
    double spare;
    bool has;
    QCB_HD LinkStream(uint64_t seed, uint32_t link_, uint32_t sweep_, uint32_t tag_)
        : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), link(link_), sweep(sweep_), tag(tag_), n(0), spare(0),
          has(false) {}
    QCB_HD double next() {
        if (has) {
            has = false;
            return spare;
        }
        uint32_t c[4] = {n, link, sweep, tag};
        philox4x32_10(c, k0, k1);
        n++;
        spare = u53(c[2], c[3]);
        has = true;
        return u53(c[0], c[1]);
    }
};

}  // namespace qcb
