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
//     on the GPU race on it and both results are undefined.  Every operator owns its own stream, so
//     two calls on DIFFERENT operators of one device overlap even when one host thread issues them
//     back to back: the host must order them (an event recorded on one operator's stream and waited
//     on by the other's, or a synchronisation) before they may share the array.  Only calls on the
//     same operator's stream are ordered by that stream.
//   - the first call on a device does the set-up: cudaGetSymbolAddress of the array with that
//     device current (it may load the module).  Make that first call before any stream capture
//     that the host starts on that device.  The address is cached per device together with the CUDA
//     context it was taken in; a call in a different context (after cudaDeviceReset, or a primary
//     context the host released and re-created) repeats the set-up, so that first call after a reset
//     must also come before any capture.
#include <mutex>
#include "common.cuh"
#include "ie_internal.h"

namespace {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kStaticScratchBytes];

std::mutex g_scratch_mu;
void *g_scratch_addr[kMaxDevices] = {};
void *g_scratch_ctx[kMaxDevices] = {};

// The driver's cuCtxGetCurrent, reached through the runtime so the library needs no link-time libcuda.
typedef int (*CtxGetCurrentFn)(void **);
CtxGetCurrentFn ctx_get_current()
{
    static CtxGetCurrentFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(p);
        tried = true;
    }
    return fn;
}

}  // namespace

int ie_static_scratch(void **ptr, size_t *capacity)
{
    *ptr = nullptr;
    *capacity = kStaticScratchBytes;
    int dev = -1;
    G2_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return G2_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    CtxGetCurrentFn get = ctx_get_current();
    if (!get) {
        g2_set_error(__FILE__, __LINE__, "cuCtxGetCurrent unavailable");
        return G2_ERR_CUDA;
    }
    void *ctx = nullptr;
    if (get(&ctx) != 0) ctx = nullptr;
    if (!ctx || !g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
        // set-up: the symbol lookup also makes the device's context current in this thread
        void *p = nullptr;
        G2_CUDA_CHECK(cudaGetSymbolAddress(&p, g_scratch));
        if (get(&ctx) != 0 || !ctx) {
            g2_set_error(__FILE__, __LINE__, "no current CUDA context after the symbol lookup");
            return G2_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
        g_scratch_ctx[dev] = ctx;
    }
    *ptr = g_scratch_addr[dev];
    return G2_OK;
}
