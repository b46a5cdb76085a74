// qcb_noalloc.cu -- mean plaquette of caller-owned device links, with no allocation at all.
//
// Some callers cannot let a library call cudaMalloc: code running inside a framework that
// owns every byte of device memory through its own pool (so a stray cudaMalloc breaks its
// accounting or fails once the pool has taken the card), hosts that forbid allocation
// after start-up, or loops that must not stall on the allocator's implicit synchronisation.
// For them qcb_plaquette_noalloc measures the plaquette of links that already sit in device
// memory and writes the result to device memory the caller provides.  The only scratch it
// needs -- one partial sum per reduction block -- lives in the fixed static device array
// below, which every GPU that loads libqcb.so holds until the process exits.
//
// Sharing and ordering rules (also stated in include/qcb.h):
//   * every call on a device uses the same array; two calls that overlap on the GPU (on
//     different streams, or on the same stream through graph branches) race on it;
//   * the array keeps the last call's contents; each call writes every slot it later reads
//     before reading it, so nothing has to start at zero;
//   * the first call on each device looks the array's device address up with
//     cudaGetSymbolAddress (with that device current) and caches it; make that first call
//     before any stream capture begins on the device.  The cached address belongs to the
//     device's current context: a cudaDeviceReset (or any other teardown of the primary
//     context) between calls is not supported, because the module may reload elsewhere.
#include <cuda_runtime.h>

#include <stdint.h>

#include <mutex>

#include "qcb_internal.h"
#include "qcb_kernels.cuh"

using namespace qcb;

namespace {

// Partial-sum slots: the plaquette reduction runs a grid of at most 148*8 blocks per parity
// (a grid-stride loop covers any lattice), so 2 * 148 * 8 doubles (18.5 KiB) always suffice.
constexpr int kNoallocPartials = 2 * 148 * 8;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoallocPartials];

std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {nullptr};

// The host-side name g_noalloc_scratch is only a stand-in: its device address is looked up
// once per device and cached.
int scratch_address(void** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(QCB_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(QCB_EINVAL, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_addr_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(QCB_ECUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return QCB_OK;
}

// Sum of nb partials in the fixed order of k_finalize, divided by 6V on the device.
__global__ void k_noalloc_final(const double* partials, int nb, double norm, double* out) {
    __shared__ double sm[256];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nb; i += 256) acc += partials[i];
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sm[0] / norm;
}

}  // namespace

extern "C" int qcb_plaquette_noalloc(const int L[4], const double* d_links, double* d_plaq, void* stream) {
    if (!L || !d_links || !d_plaq) return fail(QCB_EINVAL, "null argument");
    int64_t V = 0;
    if (!lattice_ok(L, &V)) return fail(QCB_EINVAL, "lattice extents must be even, >= 2, volume <= 2^30 sites");
    // the kernel reads the links as 16-byte (re, im) pairs and writes one double
    if (((uintptr_t)d_links & 15u) != 0) return fail(QCB_EINVAL, "d_links must be 16-byte aligned");
    if (((uintptr_t)d_plaq & 7u) != 0) return fail(QCB_EINVAL, "d_plaq must be 8-byte aligned");
    const Geom g = make_geom(L);
    const int64_t need = (g.Vh + 255) / 256;
    const unsigned nbx = (unsigned)(need < 148 * 8 ? need : 148 * 8);
    const int nb = (int)(2 * nbx);
    if (nb > kNoallocPartials)
        return fail(QCB_EINVAL, "reduction needs %d partial sums, static scratch holds %d", nb, kNoallocPartials);
    void* scratch = nullptr;
    int r = scratch_address(&scratch);
    if (r != QCB_OK) return r;
    cudaStream_t s = (cudaStream_t)stream;
    LinkField<double, 9, false> U;  // the caller's untiled layout
    U.p = (double2*)d_links;
    U.Vh = g.Vh;
    k_plaquette<double, 9, false><<<dim3(2, nbx), 256, 0, s>>>(g, U, (double*)scratch);
    k_noalloc_final<<<1, 256, 0, s>>>((const double*)scratch, nb, 6.0 * (double)V, d_plaq);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(QCB_ECUDA, "plaquette_noalloc launch: %s", cudaGetErrorString(e));
    note_launches(2);
    return QCB_OK;
}
