// Static-scratch IE apply: giem2g_apply_ie_operator_device_static.
//
// The apply needs two intermediates (U1: x-transformed vectors, Uhat: the 2-D spectrum) that the
// regular entry points take from the operator's own buffers, which giem2g_prepare_ie_kernel
// allocates.  This entry point takes them instead from one fixed array in the library's device
// image, so a call performs no device allocation of any kind: no cudaMalloc/cudaFree, no pool, no
// library that allocates.  It serves hosts that must not allocate device memory while they run:
// a host that sizes its device memory once at start-up and hands all of it to its own pool (the
// reference's host allocates its kernel and FFT buffers once, giem2g.F90:238-242, and expects
// nothing else to grow) cannot take a call-time cudaMalloc, because once its pool owns the free
// memory that cudaMalloc fails, and cudaMalloc/cudaFree also synchronise the device against the
// host's other streams.  The array is reserved when the CUDA module is loaded and never grows.
//
// Limits and rules:
//   - capacity kStaticScratchBytes (32 MiB).  The apply needs 18*Nx*Ny*Nz complex elements
//     (U1 6*Nx*Ny*Nz, Uhat 12*Nx*Ny*Nz): 16 B each for precision 0, 8 B for precision 1, so e.g.
//     64x64x16 fits at both precisions and 128x128x32 fits at neither.  Larger grids are rejected
//     with G2_ERR_ARG and a message; they keep using giem2g_apply_ie_operator_device.
//   - every call on a device shares the one array.  Nothing in it has to start at zero (every
//     element is written before it is read within a call), but two calls whose executions overlap
//     on the GPU (different streams, or different host threads, of the same device) race on it
//     and both results are undefined.  Calls on the operator's stream are ordered and safe.
//   - the first call on a device does the set-up: cudaGetSymbolAddress of the array with that
//     device current (it may load the module).  Make that first call before any stream capture
//     that the host starts on that device.
#include <mutex>
#include "common.cuh"
#include "ie_internal.h"

namespace {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kStaticScratchBytes];

std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices] = {};

}  // namespace

int ie_static_scratch(void **ptr, size_t *capacity)
{
    *ptr = nullptr;
    *capacity = kStaticScratchBytes;
    int dev = -1;
    G2_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return G2_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        G2_CUDA_CHECK(cudaGetSymbolAddress(&p, g_scratch));
        g_scratch_addr[dev] = p;
    }
    *ptr = g_scratch_addr[dev];
    return G2_OK;
}
