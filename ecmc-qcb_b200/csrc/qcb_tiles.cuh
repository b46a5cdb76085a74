// qcb_tiles.cuh -- kernels over a work list of tiles drawn from one or many lattices.
//
// A work list covers nlat lattices (the chains of a batch, the requests of a serving step, or a
// single field).  Lattice i owns nb_i = ceil(V_i / 2 / TILE) "blocks" of half-sites; a kernel
// of kind m (m = 1 heatbath, 8 flow, 2 plaquette, 6 clover) sees m * nb_i tiles for that lattice,
// stored contiguously from tile m * nb_begin_i.  tile_lat maps a block index (t / m) to its
// lattice; with a single lattice it is NULL.  Kernels are persistent: a grid sized to the
// resident capacity of the GPU walks the list with a stride of gridDim.x.
#pragma once
#include "qcb_kernels.cuh"

namespace qcb {

constexpr int TILE = 128;  // threads (half-sites) per tile in every work list

struct LatDesc {
    Geom g;
    void* links;      // heatbath: links updated in place; flow: buffer A of the ping-pong pair
    void* links_out;  // flow: buffer B of the ping-pong pair
    void* z;          // flow: su(3) accumulator (8 reals per link)
    double* meas;     // serving: per-step measurements (nv doubles per step)
    double c_alpha;   // heatbath: -0.75 / beta
    double eps;       // flow step size
    uint64_t seed;    // heatbath stream key
    int nb_begin;     // prefix sum of the nb of the lattices before this one
    int nb;           // ceil(Vh / TILE)
    int flip;         // flow: 1 if the current links sit in links_out (xor the launch's flip_xor)
    int tick0;        // serving: scheduler tick at which this lattice took its first measurement
    void* halves;     // serving: clover halves of the measuring stage 1 (halves_bytes)
};

template <typename R, int NE>
__device__ __forceinline__ LinkField<R, NE> lview(void* p, int64_t Vh) {
    LinkField<R, NE> f;
    f.p = (typename LinkField<R, NE>::C2*)p;
    f.Vh = Vh;
    return f;
}

// Descriptor of the lattice that owns block index blk: from the device array when there is one,
// else the single descriptor passed by value.
__device__ __forceinline__ const LatDesc* lattice_of(const LatDesc* lats, const int* tile_lat, const LatDesc& one,
                                                     int blk) {
    if (!lats) return &one;
    return lats + (tile_lat ? __ldg(tile_lat + blk) : 0);
}

// ---------------------------------------------------------------- heatbath, one (parity, MU) phase
// Threads walk the concatenated tiles (TILE half-sites each) in strides of the grid, so any
// BLOCK size covers the same work list.
template <typename R, int NE, int MU, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_hb_tiles(const LatDesc* __restrict__ lats, const int* __restrict__ tile_lat, const LatDesc one, int ntiles,
               int par, int n_hits, const uint32_t* sweep_dev, uint32_t sweep_add, int reproject, int* err) {
    const uint32_t sweep = sweep_add + (sweep_dev ? *sweep_dev : 0u);
    const int64_t total = (int64_t)ntiles * TILE;
    constexpr bool SLOT = HbSlotFits<R, BLOCK>::value;
    __shared__ typename V2<R>::T slot[(SLOT ? 18 : 1) * BLOCK];
    typename V2<R>::T* my = slot + threadIdx.x;
    for (int64_t v = (int64_t)blockIdx.x * BLOCK + threadIdx.x; v < total; v += (int64_t)gridDim.x * BLOCK) {
        const int tile = (int)(v / TILE);
        const LatDesc* d = lattice_of(lats, tile_lat, one, tile);
        const Geom g = d->g;
        const int h = (tile - d->nb_begin) * TILE + (int)(v % TILE);
        if (h < g.Vh)
            hb_link<R, NE, MU, SLOT>(g, lview<R, NE>(d->links, g.Vh), par, h, d->c_alpha, n_hits, d->seed, sweep,
                                     reproject, err, my, BLOCK);
    }
}

// ---------------------------------------------------------------- flow, one RK3 stage
// Tile classes interleave the 8 (mu, parity) link classes of a block of sites so that they
// share their neighbour links in L2.  With f = flip ^ flip_xor, the input of stage s is links
// when (f + s - 1) is even; a whole RK3 step therefore moves the field to the other buffer.
template <typename R, int NE, int STAGE>
__global__ void __launch_bounds__(QCB_FLOW_THREADS, QCB_FLOW_MINB(R))
    k_flow_tiles(const LatDesc* __restrict__ lats, const int* __restrict__ tile_lat, const LatDesc one, int ntiles,
                 int flip_xor, int reproject) {
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const LatDesc* d = lattice_of(lats, tile_lat, one, t >> 3);
        const Geom g = d->g;
        const int lt = t - 8 * d->nb_begin;
        const int cls = lt & 7;
        const int h = (lt >> 3) * TILE + threadIdx.x;
        if (h >= g.Vh) continue;
        const bool in_b = (((d->flip ^ flip_xor) + STAGE - 1) & 1) != 0;
        const LinkField<R, NE> win = lview<R, NE>(in_b ? d->links_out : d->links, g.Vh);
        const LinkField<R, NE> wout = lview<R, NE>(in_b ? d->links : d->links_out, g.Vh);
        AlgField<R> z;
        z.p = (typename AlgField<R>::C2*)d->z;
        z.Vh = g.Vh;
        flow_link<R, NE, STAGE>(g, win, wout, z, d->eps, cls >> 1, cls & 1, h, reproject);
    }
}

// Stage 1 that also writes each lattice's clover halves (the serving tick's measurement; see
// k_flow_stage1_meas).  The links it writes are those of k_flow_tiles<R, NE, 1>.
template <typename R, int NE>
__global__ void __launch_bounds__(QCB_FLOW_THREADS, QCB_FLOW_MEAS_MINB(R))
    k_flow_tiles1_meas(const LatDesc* __restrict__ lats, const int* __restrict__ tile_lat, const LatDesc one,
                       int ntiles, int flip_xor, int reproject) {
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const LatDesc* d = lattice_of(lats, tile_lat, one, t >> 3);
        const Geom g = d->g;
        const int lt = t - 8 * d->nb_begin;
        const int cls = lt & 7;
        const int h = (lt >> 3) * TILE + threadIdx.x;
        if (h >= g.Vh) continue;
        const bool in_b = ((d->flip ^ flip_xor) & 1) != 0;
        const LinkField<R, NE> win = lview<R, NE>(in_b ? d->links_out : d->links, g.Vh);
        const LinkField<R, NE> wout = lview<R, NE>(in_b ? d->links : d->links_out, g.Vh);
        AlgField<R> z;
        z.p = (typename AlgField<R>::C2*)d->z;
        z.Vh = g.Vh;
        const HalfClovers<R> H{(R*)d->halves, 2 * g.Vh};
        flow_link<R, NE, 1, true>(g, win, wout, z, d->eps, cls >> 1, cls & 1, h, reproject, H);
    }
}

// ---------------------------------------------------------------- per-tile reductions
// Clover halves -> (q, e) per tile: 2 tiles per lattice block of sites (one per parity), so the
// per-lattice finalize sums 2 * nb partials; the per-site values are those of k_clover_halves.
template <typename R>
__global__ void __launch_bounds__(TILE)
    k_halves_tiles(const LatDesc* __restrict__ lats, const int* __restrict__ tile_lat, const LatDesc one, int ntiles,
                   double* partials) {
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const LatDesc* d = lattice_of(lats, tile_lat, one, t >> 1);
        const int64_t Vh = d->g.Vh;
        const int lt = t - 2 * d->nb_begin;
        const int h = (lt >> 1) * TILE + threadIdx.x;
        const HalfClovers<R> H{(R*)d->halves, 2 * Vh};
        double v[3] = {0.0, 0.0, 0.0};
        if (h < Vh) site_halves_qe(H, (int64_t)(lt & 1) * Vh + h, v);
        block_sum_store<2>(v, partials, t);
        __syncthreads();
    }
}
// flip_xor < 0: measure `links`; otherwise measure the flow's current buffer (as above).
// Plaquette: 2 tiles per block (one per parity); one partial per tile.
template <typename R, int NE>
__global__ void __launch_bounds__(TILE)
    k_plaq_tiles(const LatDesc* __restrict__ lats, const int* __restrict__ tile_lat, const LatDesc one, int ntiles,
                 int flip_xor, double* partials) {
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const LatDesc* d = lattice_of(lats, tile_lat, one, t >> 1);
        const Geom g = d->g;
        const int lt = t - 2 * d->nb_begin;
        const int par = lt & 1;
        const int h = (lt >> 1) * TILE + threadIdx.x;
        void* base = (flip_xor >= 0 && (d->flip ^ flip_xor)) ? d->links_out : d->links;
        double v[1] = {h < g.Vh ? site_plaquette(g, lview<R, NE>(base, g.Vh), par, h) : 0.0};
        block_sum_store<1>(v, partials, t);
        __syncthreads();
    }
}

// Clover Q/E: 6 tiles per block (parity x plane pair); two partials (q, e) per tile.
template <typename R, int NE>
__global__ void __launch_bounds__(TILE, QCB_CLOVER_MINB(R))
    k_clover_tiles(const LatDesc* __restrict__ lats, const int* __restrict__ tile_lat, const LatDesc one, int ntiles,
                   int flip_xor, double* partials) {
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const LatDesc* d = lattice_of(lats, tile_lat, one, t / 6);
        const Geom g = d->g;
        const int lt = t - 6 * d->nb_begin;
        const int cls = lt % 6;
        const int h = (lt / 6) * TILE + threadIdx.x;
        void* base = (flip_xor >= 0 && (d->flip ^ flip_xor)) ? d->links_out : d->links;
        double v[2] = {0.0, 0.0};
        if (h < g.Vh) site_clover_pair<R, NE, 2>(g, lview<R, NE>(base, g.Vh), cls & 1, cls >> 1, h, v);
        block_sum_store<2>(v, partials, t);
        __syncthreads();
    }
}

// Per-lattice deterministic sum of the partials of its m*nb tiles (one block per lattice),
// scaled: out[i*nv + k] = scale_k(i) * sum.  scale mode 0: none; 1: plaquette 1/(6V);
// 2: clover (1, 1/V).
__global__ void k_lat_finalize(const LatDesc* __restrict__ lats, const LatDesc one, const double* __restrict__ partials,
                               int m, int nv, int scale_mode, double* out);

}  // namespace qcb
