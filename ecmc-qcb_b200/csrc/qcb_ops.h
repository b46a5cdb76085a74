// qcb_ops.h -- launchers of every kernel for one storage format, as a table of host functions.
//
// Each of the four storage formats (FP64/FP32 x 18/12 reals) is compiled in its own
// translation unit (qcb_fmt_*.cu) from the templates of qcb_fmt.cuh; the C ABI picks the table
// of a handle's format at run time.
#pragma once
#include <cuda_runtime.h>

#include "qcb_tiles.cuh"

namespace qcb {

// A work list of tiles over device-resident lattice descriptors.
struct WorkList {
    const LatDesc* lats = nullptr;  // device array of nlat descriptors; NULL: use `one`
    const int* tile_lat = nullptr;  // device map block -> lattice (NULL when nlat == 1)
    LatDesc one{};                  // the descriptor of a single lattice, passed by value
    int nb_total = 0;               // sum over lattices of ceil(Vh / TILE)
    int nlat = 0;
};

// Heatbath launch shapes the autotuner chooses among: (threads per block, min blocks per SM).
constexpr int kHbVariants = 3;

struct FmtOps {
    // ---- work-list kernels (one or many lattices)
    cudaError_t (*hb)(const WorkList& w, int variant, int par, int mu, int n_hits, const uint32_t* sweep_dev,
                      uint32_t sweep_add, int reproject, int* err, cudaStream_t s);
    cudaError_t (*flow)(const WorkList& w, int stage, int flip_xor, int reproject, cudaStream_t s);
    cudaError_t (*plaq_tiles)(const WorkList& w, int flip_xor, double* partials, cudaStream_t s);
    cudaError_t (*clover_tiles)(const WorkList& w, int flip_xor, double* partials, cudaStream_t s);
    // the tiled measuring stage 1 (clover halves into each LatDesc's `halves`) and their sums, two
    // (q, e) partials a lattice block of sites
    cudaError_t (*flow_tiles1_meas)(const WorkList& w, int flip_xor, int reproject, cudaStream_t s);
    cudaError_t (*halves_tiles)(const WorkList& w, double* partials, cudaStream_t s);
    // ---- single-lattice kernels
    cudaError_t (*hb1)(const Geom& g, void* links, int par, int mu, double c_alpha, int n_hits, uint64_t seed,
                       uint32_t sweep, int reproject, int* err, cudaStream_t s);
    cudaError_t (*hb_one)(const Geom& g, void* links, int par, int h, int mu, double c_alpha, int n_hits,
                          uint64_t seed, uint32_t sweep, int reproject, int* err, double2* a_out, cudaStream_t s);
    cudaError_t (*probe_link)(const Geom& g, const void* links, int mu, int par, int h, double* out,
                              cudaStream_t s);
    cudaError_t (*flow1)(const Geom& g, const void* win, void* wout, void* z, double eps, int stage, int reproject,
                         cudaStream_t s);
    // stage 1 that also writes the clover halves of its input (hbuf: halves_bytes), and their sum
    cudaError_t (*flow1_meas)(const Geom& g, const void* win, void* wout, void* z, double eps, int reproject,
                              void* hbuf, cudaStream_t s);
    cudaError_t (*clover_halves)(const Geom& g, const void* hbuf, double* partials, unsigned nb, cudaStream_t s);
    cudaError_t (*flow_force)(const Geom& g, const void* w, void* f, cudaStream_t s);
    cudaError_t (*flow_update)(const Geom& g, void* w, const void* f0, const void* f1, double a, double b, int use_f1,
                               int reproject, cudaStream_t s);
    cudaError_t (*flow_replace)(const Geom& g, void* f0, const void* f1, cudaStream_t s);
    cudaError_t (*clover_site)(const Geom& g, const void* links, int par, int h, int mu, int nu, double* out,
                               cudaStream_t s);
    cudaError_t (*plaquette)(const Geom& g, const void* links, double* partials, unsigned nbx, cudaStream_t s);
    cudaError_t (*clover)(const Geom& g, const void* links, double* partials, unsigned nbx, cudaStream_t s);
    cudaError_t (*unitarity)(const Geom& g, const void* links, double* partials, unsigned nbx, cudaStream_t s);
    cudaError_t (*aos_to_soa)(const Geom& g, const double2* aos, void* links, int bswap, cudaStream_t s);
    cudaError_t (*soa_to_aos)(const Geom& g, const void* links, double2* aos, int bswap, cudaStream_t s);
    cudaError_t (*start)(const Geom& g, void* links, int hot, uint64_t seed, cudaStream_t s);
    cudaError_t (*shift)(const Geom& g, const void* src, void* dst, const int sh[4], cudaStream_t s);
    cudaError_t (*reunitarize)(const Geom& g, void* links, cudaStream_t s);
    cudaError_t (*staple_field)(const Geom& g, const void* links, int mu, double2* out, cudaStream_t s);
    const char* hb_variant_name[kHbVariants];
};

extern const FmtOps kOpsD18, kOpsD12, kOpsF18, kOpsF12;

inline const FmtOps& fmt_ops(int fmt) {
    switch (fmt) {
        case 0: return kOpsD18;
        case 1: return kOpsD12;
        case 2: return kOpsF18;
        default: return kOpsF12;
    }
}

// Streaming multiprocessors of the current device (cached).
int sm_count();

}  // namespace qcb
