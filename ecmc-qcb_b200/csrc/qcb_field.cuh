// qcb_field.cuh -- lattice geometry, parity-split SoA link storage and the Philox link streams.
//
// Geometry follows the reference's GeometryCB conventions (src/geometry/GeometryCB.h:25-27,
// GeometryCB.cpp:57-67): lexicographic site index with x fastest and t slowest, direction
// order mu = x,y,z,t, site parity (x+y+z+t) mod 2.  The reference's (L+2)^4 halo box, its
// neighbour table and frozen-link mask are replaced by periodic coordinate arithmetic on a
// single periodic lattice: one GPU holds the whole lattice, so there is no halo to refresh.
//
// HBM layout of one field ("parity-split, tiled structure of arrays"):
//     plane(mu, parity) = mu*2 + parity, tile = h / 32, lane = h % 32  (h = lex/2)
//     element e of link (mu, parity, h) = base[((plane * nT + tile) * NE + e) * 32 + lane]
// with one complex per element and nT = ceil(V/2 / 32) (FP32 tiles pair the elements into 128-bit
// words, see LinkField).  Lx is even, so the two sites 2k, 2k+1 of an x-row have opposite parity
// and share h = k.  A warp of 32 consecutive h reads one contiguous run per element (or element
// pair), and the elements of one link sit at compile-time offsets from one base address, so a
// link load costs one address computation.  NE = 9 stores the full matrix (18 reals); NE = 6 the
// first two rows (12 reals), the third rebuilt in registers as conj(row0 x row1).
// The untiled variant (TILED = false: element e at base[(plane*NE + e)*V/2 + h]) is the layout of
// caller-owned links handed to the allocation-free entry point.
#pragma once
#include <stdint.h>

#include "qcb_su3.cuh"

namespace qcb {

#ifdef QCB_CHECKED
// Checked build (libqcb_checked.so): every (mu, parity, h) that a link or algebra access is
// formed from is validated on the device before the address is.  A bad one is counted in this
// translation unit's record, the first is kept as kind << 62 | (mu & 63) << 56 | (par & 255) << 48
// | (h mod 2^48) (kind 0 = link, 1 = su(3) algebra, 2 = clover halves: mu = the real mod 64, parity = 1 past the
// sites), and the access is redirected to link
// (0, 0, 0), inside the allocation, so the kernel runs on instead of faulting.  The host reads
// and clears every translation unit's record through qcb_debug_oob.
static __device__ unsigned long long g_oob_count;
static __device__ unsigned long long g_oob_first;
static __device__ __noinline__ void note_oob(int kind, int mu, int par, int64_t h) {
    const unsigned long long key = ((unsigned long long)kind << 62) | ((unsigned long long)(mu & 63) << 56) |
                                   ((unsigned long long)(par & 255) << 48) |
                                   ((unsigned long long)h & 0xFFFFFFFFFFFFull);
    if (atomicAdd(&g_oob_count, 1ull) == 0ull) g_oob_first = key;
}
typedef cudaError_t (*OobTake)(unsigned long long* count, unsigned long long* first);
void register_oob(OobTake fn);  // the registry lives in qcb_api.cu
// This translation unit's record, read and cleared (invalid-symbol when the unit has no kernels).
static cudaError_t oob_take(unsigned long long* count, unsigned long long* first) {
    cudaError_t e = cudaMemcpyFromSymbol(count, g_oob_count, sizeof(*count));
    if (e == cudaSuccess) e = cudaMemcpyFromSymbol(first, g_oob_first, sizeof(*first));
    const unsigned long long zero = 0;
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_oob_count, &zero, sizeof(zero));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_oob_first, &zero, sizeof(zero));
    return e;
}
static const int g_oob_registered = (register_oob(&oob_take), 0);
#endif

// Validates (mu, par, h) of a field access in the checked build (see above); a no-op otherwise.
QCB_HD void check_index(int kind, int& mu, int& par, int& h, int64_t Vh) {
#if defined(QCB_CHECKED) && defined(__CUDA_ARCH__)
    if (!((unsigned)mu < 4u && (unsigned)par < 2u && h >= 0 && (int64_t)h < Vh)) {
        note_oob(kind, mu, par, h);
        mu = 0;
        par = 0;
        h = 0;
    }
#else
    (void)kind, (void)mu, (void)par, (void)h, (void)Vh;
#endif
}

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

// Division of 32-bit unsigned integers by an invariant divisor d (Granlund & Montgomery, "Division
// by invariant integers using multiplication", PLDI 1994): q = (t + ((n - t) >> 1)) >> (l - 1),
// t = mulhi(n, m), l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1; d = 1 returns n.
struct FastDiv {
    uint32_t d, m, s;
};
inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f;
    f.d = d;
    if (d <= 1) {
        f.m = 0;
        f.s = 0;
        return f;
    }
    uint32_t l = 0;
    while ((1ull << l) < d) l++;
    f.m = (uint32_t)((((1ull << 32) * ((1ull << l) - d)) / d) + 1);
    f.s = l;
    return f;
}
QCB_HD uint32_t fdiv(uint32_t n, const FastDiv& f) {
    if (f.d <= 1) return n;
#ifdef __CUDA_ARCH__
    const uint32_t t = __umulhi(n, f.m);
#else
    const uint32_t t = (uint32_t)(((uint64_t)n * f.m) >> 32);
#endif
    return (t + ((n - t) >> 1)) >> (f.s - 1);
}

struct Geom {
    int L[4];
    int stride[4];  // lexicographic strides (1, Lx, Lx*Ly, Lx*Ly*Lz)
    FastDiv div[3];  // division by L[0], L[1], L[2]
    int64_t V, Vh;
    int nT;  // 32-site tiles per parity: ceil(Vh / 32)
};

inline Geom make_geom(const int L[4]) {
    Geom g;
    for (int d = 0; d < 4; d++) g.L[d] = L[d];
    g.stride[0] = 1;
    g.stride[1] = L[0];
    g.stride[2] = L[0] * L[1];
    g.stride[3] = L[0] * L[1] * L[2];
    for (int d = 0; d < 3; d++) g.div[d] = make_fastdiv((uint32_t)L[d]);
    g.V = (int64_t)L[0] * L[1] * L[2] * L[3];
    g.Vh = g.V / 2;
    g.nT = (int)((g.Vh + 31) / 32);
    return g;
}

// Coordinates of half-site h of the given parity (lexicographic index 2h or 2h+1; V <= 2^30).
QCB_HD void site_coords(const Geom& g, int par, uint32_t h, int c[4]) {
    const uint32_t i = 2u * h;
    const uint32_t q0 = fdiv(i, g.div[0]);
    const uint32_t q1 = fdiv(q0, g.div[1]);
    const uint32_t q2 = fdiv(q1, g.div[2]);
    c[0] = (int)(i - q0 * (uint32_t)g.L[0]);
    c[1] = (int)(q0 - q1 * (uint32_t)g.L[1]);
    c[2] = (int)(q1 - q2 * (uint32_t)g.L[2]);
    c[3] = (int)q2;
    c[0] += (c[1] + c[2] + c[3] + par) & 1;
}
QCB_HD int lex_of(const Geom& g, const int c[4]) {
    return c[0] + c[1] * g.stride[1] + c[2] * g.stride[2] + c[3] * g.stride[3];
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
QCB_HD int step_up(const Geom& g, int lex, int cd, int d) {
    return (cd == g.L[d] - 1) ? lex - (g.L[d] - 1) * g.stride[d] : lex + g.stride[d];
}
QCB_HD int step_dn(const Geom& g, int lex, int cd, int d) {
    return (cd == 0) ? lex + (g.L[d] - 1) * g.stride[d] : lex - g.stride[d];
}

// Lexicographic offsets of the eight periodic neighbours of one site, held in registers so that
// code with a runtime direction selects them (sel4) instead of indexing the geometry or the
// coordinate array, which would move both into local memory.
struct Steps {
    int up[4], dn[4];
};
QCB_HD Steps make_steps(const Geom& g, const int c[4]) {
    Steps s;
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const int wrap = (g.L[d] - 1) * g.stride[d];
        s.up[d] = (c[d] == g.L[d] - 1) ? -wrap : g.stride[d];
        s.dn[d] = (c[d] == 0) ? wrap : -g.stride[d];
    }
    return s;
}
QCB_HD int sel4(const int v[4], int i) { return i == 0 ? v[0] : (i == 1 ? v[1] : (i == 2 ? v[2] : v[3])); }

// Link storage view; NE = 9 (18 reals) or 6 (12 reals, third row rebuilt on load).
//
// Tiled layout: the links of one (mu, parity) plane are cut into tiles of 32 consecutive
// half-lattice sites; a tile holds NE complex elements of its 32 links, element-major, so a
// warp reading one element of 32 neighbouring links touches one contiguous run.
//   double: element e of lane l at tile start + e*32 + l (one 128-bit double2 per access);
//   float:  elements (2k, 2k+1) of lane l as one float4 at tile start + k*64 + 2l, and for odd
//           NE the last element as a float2 at tile start + (NE-1)*32 + l, so every access but
//           that one is 128 bits wide.
// Untiled layout (caller-owned fields): element e of link (mu, par, h) at ((mu*2+par)*NE+e)*Vh+h.
template <typename R, int NE, bool TILED = true>
struct LinkField {
    typedef typename V2<R>::T C2;
    C2* p;
    int64_t Vh;
    static constexpr bool kQuad = TILED && sizeof(R) == 4;
    static constexpr int kPairs = kQuad ? NE / 2 : 0;
    // start of the tile holding link (mu, par, h)
    QCB_HD size_t tile0(int mu, int par, int h) const {
        check_index(0, mu, par, h, Vh);
        const int nT = (int)((Vh + 31) >> 5);
        return (size_t)((mu * 2 + par) * nT + (h >> 5)) * (NE * 32);
    }
    // element 0 of link (mu, par, h) for the 64-bit-element layouts; element e at + e * es()
    QCB_HD int64_t es() const { return TILED ? 32 : Vh; }
    QCB_HD size_t index0(int mu, int par, int h) const {
        if (TILED) return tile0(mu, par, h) + (h & 31);
        check_index(0, mu, par, h, Vh);
        return (size_t)((mu * 2 + par) * NE) * (size_t)Vh + (size_t)h;
    }
    template <bool RO>
    __device__ __forceinline__ static C2 rd(const C2* a) {
        if (RO) return __ldg(a);
        return *a;
    }
    template <bool RO>
    __device__ __forceinline__ M3<R> load_t(int mu, int par, int h) const {
        M3<R> u;
        if constexpr (kQuad) {
            const C2* t = p + tile0(mu, par, h);
            const float4* q = reinterpret_cast<const float4*>(t) + (h & 31);
#pragma unroll
            for (int k = 0; k < kPairs; k++) {
                const float4 v = RO ? __ldg(q + 32 * k) : q[32 * k];
                u.e[2 * k] = mkc<R>(v.x, v.y);
                u.e[2 * k + 1] = mkc<R>(v.z, v.w);
            }
            if (NE & 1) {
                const C2 v = rd<RO>(t + (NE - 1) * 32 + (h & 31));
                u.e[NE - 1] = mkc<R>(v.x, v.y);
            }
        } else {
            const C2* b = p + index0(mu, par, h);
#pragma unroll
            for (int e = 0; e < NE; e++) {
                const C2 v = rd<RO>(b + e * es());
                u.e[e] = mkc<R>(v.x, v.y);
            }
        }
        if (NE == 6) rebuild_row2(u);
        return u;
    }
    __device__ __forceinline__ M3<R> load(int mu, int par, int h) const { return load_t<false>(mu, par, h); }
    // read-only path for links that no thread of the running kernel writes
    __device__ __forceinline__ M3<R> load_ro(int mu, int par, int h) const { return load_t<true>(mu, par, h); }
    __device__ __forceinline__ void store(int mu, int par, int h, const M3<R>& u) const {
        if constexpr (kQuad) {
            C2* t = p + tile0(mu, par, h);
            float4* q = reinterpret_cast<float4*>(t) + (h & 31);
#pragma unroll
            for (int k = 0; k < kPairs; k++)
                q[32 * k] = make_float4(u.e[2 * k].re, u.e[2 * k].im, u.e[2 * k + 1].re, u.e[2 * k + 1].im);
            if (NE & 1) {
                C2 v;
                v.x = u.e[NE - 1].re;
                v.y = u.e[NE - 1].im;
                t[(NE - 1) * 32 + (h & 31)] = v;
            }
        } else {
            C2* b = p + index0(mu, par, h);
#pragma unroll
            for (int e = 0; e < NE; e++) {
                C2 v;
                v.x = u.e[e].re;
                v.y = u.e[e].im;
                b[e * es()] = v;
            }
        }
    }
    // raw element copy of one link (no rebuild / re-encode for NE == 6)
    __device__ __forceinline__ void copy_from(int mu, int par, int h, const LinkField& src, int spar, int sh) const {
        if constexpr (kQuad) {
            C2* t = p + tile0(mu, par, h);
            const C2* a = src.p + src.tile0(mu, spar, sh);
            float4* q = reinterpret_cast<float4*>(t) + (h & 31);
            const float4* r = reinterpret_cast<const float4*>(a) + (sh & 31);
#pragma unroll
            for (int k = 0; k < kPairs; k++) q[32 * k] = __ldg(r + 32 * k);
            if (NE & 1) t[(NE - 1) * 32 + (h & 31)] = __ldg(a + (NE - 1) * 32 + (sh & 31));
        } else {
            C2* b = p + index0(mu, par, h);
            const C2* a = src.p + src.index0(mu, spar, sh);
#pragma unroll
            for (int e = 0; e < NE; e++) b[e * es()] = __ldg(a + e * src.es());
        }
    }
};

// su(3) algebra storage: 8 reals per link as 4 complex entries, tiled like LinkField
//   0: Z01, 1: Z02, 2: Z12, 3: (Im Z00, Im Z11);  Z22 = -i(Im Z00 + Im Z11), Zji = -conj(Zij).
// double: entry k of lane l at tile start + k*32 + l; float: entries (0,1) as one float4 at
// tile start + 2l and entries (2,3) at tile start + 64 + 2l.
template <typename R>
struct AlgField {
    typedef typename V2<R>::T C2;
    static constexpr bool kQuad = sizeof(R) == 4;
    C2* p;
    int64_t Vh;
    QCB_HD size_t tile0(int mu, int par, int h) const {
        check_index(1, mu, par, h, Vh);
        const int nT = (int)((Vh + 31) >> 5);
        return (size_t)((mu * 2 + par) * nT + (h >> 5)) * (4 * 32);
    }
    __device__ __forceinline__ M3<R> load(int mu, int par, int h) const {
        C2 z01, z02, z12, dg;
        if constexpr (kQuad) {
            const float4* q = reinterpret_cast<const float4*>(p + tile0(mu, par, h)) + (h & 31);
            const float4 a = q[0], b = q[32];
            z01 = make_float2(a.x, a.y);
            z02 = make_float2(a.z, a.w);
            z12 = make_float2(b.x, b.y);
            dg = make_float2(b.z, b.w);
        } else {
            const C2* b = p + tile0(mu, par, h) + (h & 31);
            z01 = b[0];
            z02 = b[32];
            z12 = b[64];
            dg = b[96];
        }
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
    __device__ __forceinline__ void store(int mu, int par, int h, const M3<R>& z) const {
        if constexpr (kQuad) {
            float4* q = reinterpret_cast<float4*>(p + tile0(mu, par, h)) + (h & 31);
            q[0] = make_float4(z(0, 1).re, z(0, 1).im, z(0, 2).re, z(0, 2).im);
            q[32] = make_float4(z(1, 2).re, z(1, 2).im, z(0, 0).im, z(1, 1).im);
        } else {
            C2* b = p + tile0(mu, par, h) + (h & 31);
            C2 v;
            v.x = z(0, 1).re;
            v.y = z(0, 1).im;
            b[0] = v;
            v.x = z(0, 2).re;
            v.y = z(0, 2).im;
            b[32] = v;
            v.x = z(1, 2).re;
            v.y = z(1, 2).im;
            b[64] = v;
            v.x = z(0, 0).im;
            v.y = z(1, 1).im;
            b[96] = v;
        }
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
        // separate high and low products (faster here than one 32x32 -> 64-bit product: a
        // 32^4 FP64 heatbath sub-sweep takes 0.206 ms against 0.213 ms)
        const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
        const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
#else
        const uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
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
// (Forming the parts of Philox rounds 0 and 1 that do not depend on the call index once per link
// was measured slower: 0.211 against 0.208 ms a 32^4 FP64 sub-sweep, 0.172 against 0.163 ms FP32.)
struct LinkStream {
    uint32_t k0, k1, link, sweep, tag, n;
    double spare;
    bool has;
    QCB_HD LinkStream(uint64_t seed, uint32_t link_, uint32_t sweep_, uint32_t tag_)
        : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), link(link_), sweep(sweep_), tag(tag_), n(0), spare(0),
          has(false) {}
    // The two doubles of Philox call n, (u53(w0, w1), u53(w2, w3)): draws 2n and 2n+1 of the
    // stream, without touching the stream's position.
    QCB_HD double2 call(uint32_t n_) const {
        uint32_t c[4] = {n_, link, sweep, tag};
        philox4x32_10(c, k0, k1);
        double2 r;
        r.x = u53(c[0], c[1]);
        r.y = u53(c[2], c[3]);
        return r;
    }
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
