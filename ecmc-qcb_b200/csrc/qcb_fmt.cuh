// qcb_fmt.cuh -- launcher implementations for one storage format (included once per format).
#pragma once
#include <algorithm>

#include "qcb_ops.h"

namespace qcb {

template <typename R, int NE>
struct FmtImpl {
    static LinkField<R, NE> view(const void* p, int64_t Vh) {
        LinkField<R, NE> f;
        f.p = (typename LinkField<R, NE>::C2*)p;
        f.Vh = Vh;
        return f;
    }

    // Resident-grid size of a persistent kernel: blocks per SM (occupancy) x SMs, cached per
    // kernel instance.
    template <typename K>
    static int resident_blocks(K kernel, int block, int* cache) {
        if (*cache == 0) {
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1)
                per_sm = 1;
            *cache = per_sm * sm_count();
        }
        return *cache;
    }

    template <int MU, int BLOCK, int MINB>
    static cudaError_t hb_launch(const WorkList& w, int par, int n_hits, const uint32_t* sweep_dev, uint32_t sweep_add,
                                 int reproject, int* err, cudaStream_t s) {
        static int cache = 0;
        auto k = k_hb_tiles<R, NE, MU, BLOCK, MINB>;
        const int64_t need = ((int64_t)w.nb_total * TILE + BLOCK - 1) / BLOCK;
        const int grid = (int)std::min<int64_t>(need, resident_blocks(k, BLOCK, &cache));
        k<<<grid, BLOCK, 0, s>>>(w.lats, w.tile_lat, w.one, w.nb_total, par, n_hits, sweep_dev, sweep_add, reproject, err);
        return cudaGetLastError();
    }
    template <int MU>
    static cudaError_t hb_mu(const WorkList& w, int variant, int par, int n_hits, const uint32_t* sd, uint32_t sa,
                             int rep, int* err, cudaStream_t s) {
        constexpr bool f64 = sizeof(R) == 8;
        switch (variant) {
            case 0: return hb_launch<MU, 64, f64 ? 8 : 12>(w, par, n_hits, sd, sa, rep, err, s);
            case 2: return hb_launch<MU, 256, 2>(w, par, n_hits, sd, sa, rep, err, s);
            default: return hb_launch<MU, 128, f64 ? 4 : 6>(w, par, n_hits, sd, sa, rep, err, s);
        }
    }
    static cudaError_t hb(const WorkList& w, int variant, int par, int mu, int n_hits, const uint32_t* sd, uint32_t sa,
                          int rep, int* err, cudaStream_t s) {
        switch (mu) {
            case 0: return hb_mu<0>(w, variant, par, n_hits, sd, sa, rep, err, s);
            case 1: return hb_mu<1>(w, variant, par, n_hits, sd, sa, rep, err, s);
            case 2: return hb_mu<2>(w, variant, par, n_hits, sd, sa, rep, err, s);
            default: return hb_mu<3>(w, variant, par, n_hits, sd, sa, rep, err, s);
        }
    }

    template <int STAGE>
    static cudaError_t flow_launch(const WorkList& w, int flip_xor, int rep, cudaStream_t s) {
        static int cache = 0;
        auto k = k_flow_tiles<R, NE, STAGE>;
        const int ntiles = 8 * w.nb_total;
        const int grid = std::min(ntiles, resident_blocks(k, QCB_FLOW_THREADS, &cache));
        k<<<grid, QCB_FLOW_THREADS, 0, s>>>(w.lats, w.tile_lat, w.one, ntiles, flip_xor, rep);
        return cudaGetLastError();
    }
    static cudaError_t flow(const WorkList& w, int stage, int flip_xor, int rep, cudaStream_t s) {
        if (stage == 1) return flow_launch<1>(w, flip_xor, rep, s);
        if (stage == 2) return flow_launch<2>(w, flip_xor, rep, s);
        return flow_launch<3>(w, flip_xor, rep, s);
    }

    template <int MU>
    static cudaError_t hb1_mu(const Geom& g, void* links, int par, double c_alpha, int n_hits, uint64_t seed,
                              uint32_t sweep, int rep, int* err, cudaStream_t s) {
        const unsigned nb = (unsigned)((g.Vh + QCB_HB_THREADS - 1) / QCB_HB_THREADS);
        k_hb_subsweep<R, NE, MU><<<nb, QCB_HB_THREADS, 0, s>>>(g, view(links, g.Vh), par, c_alpha, n_hits, seed, sweep,
                                                               rep, err);
        return cudaGetLastError();
    }
    static cudaError_t hb1(const Geom& g, void* links, int par, int mu, double c_alpha, int n_hits, uint64_t seed,
                           uint32_t sweep, int rep, int* err, cudaStream_t s) {
        switch (mu) {
            case 0: return hb1_mu<0>(g, links, par, c_alpha, n_hits, seed, sweep, rep, err, s);
            case 1: return hb1_mu<1>(g, links, par, c_alpha, n_hits, seed, sweep, rep, err, s);
            case 2: return hb1_mu<2>(g, links, par, c_alpha, n_hits, seed, sweep, rep, err, s);
            default: return hb1_mu<3>(g, links, par, c_alpha, n_hits, seed, sweep, rep, err, s);
        }
    }
    static cudaError_t hb_one(const Geom& g, void* links, int par, int h, int mu, double c_alpha, int n_hits,
                              uint64_t seed, uint32_t sweep, int rep, int* err, double2* a_out, cudaStream_t s) {
        auto U = view(links, g.Vh);
        switch (mu) {
            case 0: k_hb_one<R, NE, 0><<<1, 1, 0, s>>>(g, U, par, h, c_alpha, n_hits, seed, sweep, rep, err, a_out); break;
            case 1: k_hb_one<R, NE, 1><<<1, 1, 0, s>>>(g, U, par, h, c_alpha, n_hits, seed, sweep, rep, err, a_out); break;
            case 2: k_hb_one<R, NE, 2><<<1, 1, 0, s>>>(g, U, par, h, c_alpha, n_hits, seed, sweep, rep, err, a_out); break;
            default: k_hb_one<R, NE, 3><<<1, 1, 0, s>>>(g, U, par, h, c_alpha, n_hits, seed, sweep, rep, err, a_out); break;
        }
        return cudaGetLastError();
    }
    static cudaError_t probe_link(const Geom& g, const void* links, int mu, int par, int h, double* out,
                                  cudaStream_t s) {
        k_probe_link<R, NE><<<1, 1, 0, s>>>(view(links, g.Vh), mu, par, h, out);
        return cudaGetLastError();
    }
    static cudaError_t flow1(const Geom& g, const void* win, void* wout, void* z, double eps, int stage, int rep,
                             cudaStream_t s) {
        const unsigned nb = 8u * (unsigned)((g.Vh + QCB_FLOW1_THREADS - 1) / QCB_FLOW1_THREADS);
        AlgField<R> za;
        za.p = (typename AlgField<R>::C2*)z;
        za.Vh = g.Vh;
        if (stage == 1)
            k_flow_stage<R, NE, 1><<<nb, QCB_FLOW1_THREADS, 0, s>>>(g, view(win, g.Vh), view(wout, g.Vh), za, eps, rep);
        else if (stage == 2)
            k_flow_stage<R, NE, 2><<<nb, QCB_FLOW1_THREADS, 0, s>>>(g, view(win, g.Vh), view(wout, g.Vh), za, eps, rep);
        else
            k_flow_stage<R, NE, 3><<<nb, QCB_FLOW1_THREADS, 0, s>>>(g, view(win, g.Vh), view(wout, g.Vh), za, eps, rep);
        return cudaGetLastError();
    }

    static cudaError_t flow1_meas(const Geom& g, const void* win, void* wout, void* z, double eps, int rep,
                                  void* hbuf, cudaStream_t s) {
        const unsigned nb = 8u * (unsigned)((g.Vh + QCB_FLOW1_THREADS - 1) / QCB_FLOW1_THREADS);
        AlgField<R> za;
        za.p = (typename AlgField<R>::C2*)z;
        za.Vh = g.Vh;
        const HalfClovers<R> H{(R*)hbuf, 2 * g.Vh};
        k_flow_stage1_meas<R, NE><<<nb, QCB_FLOW1_THREADS, 0, s>>>(g, view(win, g.Vh), view(wout, g.Vh), za, eps,
                                                                   rep, H);
        return cudaGetLastError();
    }
    static cudaError_t clover_halves(const Geom& g, const void* hbuf, double* partials, unsigned nb, cudaStream_t s) {
        const HalfClovers<R> H{(R*)hbuf, 2 * g.Vh};
        k_clover_halves<R><<<nb, 128, 0, s>>>(g, H, partials);
        return cudaGetLastError();
    }

    static AlgField<R> alg(const void* p, int64_t Vh) {
        AlgField<R> z;
        z.p = (typename AlgField<R>::C2*)p;
        z.Vh = Vh;
        return z;
    }
    static cudaError_t flow_force(const Geom& g, const void* w, void* f, cudaStream_t s) {
        const unsigned nb = 8u * (unsigned)((g.Vh + QCB_FLOW1_THREADS - 1) / QCB_FLOW1_THREADS);
        k_flow_force<R, NE><<<nb, QCB_FLOW1_THREADS, 0, s>>>(g, view(w, g.Vh), alg(f, g.Vh));
        return cudaGetLastError();
    }
    static cudaError_t flow_update(const Geom& g, void* w, const void* f0, const void* f1, double a, double b,
                                   int use_f1, int rep, cudaStream_t s) {
        const dim3 grid((unsigned)((g.Vh + 255) / 256), 8);
        k_flow_update<R, NE><<<grid, 256, 0, s>>>(g, view(w, g.Vh), alg(f0, g.Vh), alg(f1 ? f1 : f0, g.Vh), a, b,
                                                  use_f1, rep);
        return cudaGetLastError();
    }
    static cudaError_t flow_replace(const Geom& g, void* f0, const void* f1, cudaStream_t s) {
        const dim3 grid((unsigned)((g.Vh + 255) / 256), 8);
        k_flow_replace<R><<<grid, 256, 0, s>>>(g.Vh, alg(f0, g.Vh), alg(f1, g.Vh));
        return cudaGetLastError();
    }
    static cudaError_t clover_site(const Geom& g, const void* links, int par, int h, int mu, int nu, double* out,
                                   cudaStream_t s) {
        k_clover_site<R, NE><<<1, 1, 0, s>>>(g, view(links, g.Vh), par, h, mu, nu, out);
        return cudaGetLastError();
    }

    // Reduction work lists are not persistent: one block per tile, one partial per tile.
    static cudaError_t plaq_tiles(const WorkList& w, int flip_xor, double* partials, cudaStream_t s) {
        const int ntiles = 2 * w.nb_total;
        k_plaq_tiles<R, NE><<<ntiles, TILE, 0, s>>>(w.lats, w.tile_lat, w.one, ntiles, flip_xor, partials);
        return cudaGetLastError();
    }
    static cudaError_t clover_tiles(const WorkList& w, int flip_xor, double* partials, cudaStream_t s) {
        const int ntiles = 6 * w.nb_total;
        k_clover_tiles<R, NE><<<ntiles, TILE, 0, s>>>(w.lats, w.tile_lat, w.one, ntiles, flip_xor, partials);
        return cudaGetLastError();
    }

    static cudaError_t flow_tiles1_meas(const WorkList& w, int flip_xor, int rep, cudaStream_t s) {
        static int cache = 0;
        auto k = k_flow_tiles1_meas<R, NE>;
        const int ntiles = 8 * w.nb_total;
        const int grid = std::min(ntiles, resident_blocks(k, QCB_FLOW_THREADS, &cache));
        k<<<grid, QCB_FLOW_THREADS, 0, s>>>(w.lats, w.tile_lat, w.one, ntiles, flip_xor, rep);
        return cudaGetLastError();
    }
    static cudaError_t halves_tiles(const WorkList& w, double* partials, cudaStream_t s) {
        const int ntiles = 2 * w.nb_total;
        k_halves_tiles<R><<<ntiles, TILE, 0, s>>>(w.lats, w.tile_lat, w.one, ntiles, partials);
        return cudaGetLastError();
    }

    static cudaError_t plaquette(const Geom& g, const void* links, double* partials, unsigned nbx, cudaStream_t s) {
        k_plaquette<R, NE><<<dim3(2, nbx), 256, 0, s>>>(g, view(links, g.Vh), partials);
        return cudaGetLastError();
    }
    static cudaError_t clover(const Geom& g, const void* links, double* partials, unsigned nbx, cudaStream_t s) {
        k_clover_qe<R, NE><<<dim3(6, nbx), 128, 0, s>>>(g, view(links, g.Vh), partials);
        return cudaGetLastError();
    }
    static cudaError_t unitarity(const Geom& g, const void* links, double* partials, unsigned nbx, cudaStream_t s) {
        k_unitarity<R, NE><<<dim3(nbx, 8), 256, 0, s>>>(g, view(links, g.Vh), partials);
        return cudaGetLastError();
    }
    static cudaError_t aos_to_soa(const Geom& g, const double2* aos, void* links, int bswap, cudaStream_t s) {
        const unsigned nb = (unsigned)((g.V * 4 + 255) / 256);
        k_aos_to_soa<R, NE><<<nb, 256, 0, s>>>(g, aos, view(links, g.Vh), bswap);
        return cudaGetLastError();
    }
    static cudaError_t soa_to_aos(const Geom& g, const void* links, double2* aos, int bswap, cudaStream_t s) {
        const unsigned nb = (unsigned)((g.V * 4 + 255) / 256);
        k_soa_to_aos<R, NE><<<nb, 256, 0, s>>>(g, view(links, g.Vh), aos, bswap);
        return cudaGetLastError();
    }
    static cudaError_t start(const Geom& g, void* links, int hot, uint64_t seed, cudaStream_t s) {
        k_start<R, NE><<<dim3((unsigned)((g.Vh + 127) / 128), 8), 128, 0, s>>>(g, view(links, g.Vh), hot, seed);
        return cudaGetLastError();
    }
    static cudaError_t shift(const Geom& g, const void* src, void* dst, const int sh[4], cudaStream_t s) {
        k_shift<R, NE><<<dim3((unsigned)((g.Vh + 127) / 128), 8), 128, 0, s>>>(g, view(src, g.Vh), view(dst, g.Vh),
                                                                               sh[0], sh[1], sh[2], sh[3]);
        return cudaGetLastError();
    }
    static cudaError_t reunitarize(const Geom& g, void* links, cudaStream_t s) {
        k_reunitarize<R, NE><<<dim3((unsigned)((g.Vh + 127) / 128), 8), 128, 0, s>>>(g, view(links, g.Vh));
        return cudaGetLastError();
    }
    static cudaError_t staple_field(const Geom& g, const void* links, int mu, double2* out, cudaStream_t s) {
        const dim3 grid((unsigned)((g.Vh + 127) / 128), 2);
        switch (mu) {
            case 0: k_staple_field<R, NE, 0><<<grid, 128, 0, s>>>(g, view(links, g.Vh), out); break;
            case 1: k_staple_field<R, NE, 1><<<grid, 128, 0, s>>>(g, view(links, g.Vh), out); break;
            case 2: k_staple_field<R, NE, 2><<<grid, 128, 0, s>>>(g, view(links, g.Vh), out); break;
            default: k_staple_field<R, NE, 3><<<grid, 128, 0, s>>>(g, view(links, g.Vh), out); break;
        }
        return cudaGetLastError();
    }

    static FmtOps make() {
        FmtOps o;
        o.hb = &hb;
        o.flow = &flow;
        o.plaq_tiles = &plaq_tiles;
        o.clover_tiles = &clover_tiles;
        o.hb1 = &hb1;
        o.hb_one = &hb_one;
        o.probe_link = &probe_link;
        o.flow1 = &flow1;
        o.flow1_meas = &flow1_meas;
        o.flow_tiles1_meas = &flow_tiles1_meas;
        o.halves_tiles = &halves_tiles;
        o.clover_halves = &clover_halves;
        o.flow_force = &flow_force;
        o.flow_update = &flow_update;
        o.flow_replace = &flow_replace;
        o.clover_site = &clover_site;
        o.plaquette = &plaquette;
        o.clover = &clover;
        o.unitarity = &unitarity;
        o.aos_to_soa = &aos_to_soa;
        o.soa_to_aos = &soa_to_aos;
        o.start = &start;
        o.shift = &shift;
        o.reunitarize = &reunitarize;
        o.staple_field = &staple_field;
        constexpr bool f64 = sizeof(R) == 8;
        o.hb_variant_name[0] = f64 ? "64x8" : "64x12";
        o.hb_variant_name[1] = f64 ? "128x4" : "128x6";
        o.hb_variant_name[2] = "256x2";
        return o;
    }
};

}  // namespace qcb
