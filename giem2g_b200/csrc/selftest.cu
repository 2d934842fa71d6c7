// Failure-detection self-test: a wait that nothing completes must end with an error status, not a hang.
// Every spin of the library's kernels (the contraction's mbarrier ring, the tcgen05 GEMM's commits) goes
// through mbar_wait_bounded, which gives up after its limit, records a code in a device error word and
// returns; this kernel runs that wait on an mbarrier that no thread or copy ever arrives on.
#include "common.cuh"
#include "ie_internal.h"
#include "tma.cuh"

namespace {
__global__ void k_wait_unarrived(int *err, unsigned long long limit_ns)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_wait_bounded(&bar, 0, err, 77, limit_ns);
}
}  // namespace

extern "C" int giem2g_selftest_bounded_wait(int limit_ms)
{
    if (limit_ms < 1 || limit_ms > 2000) return G2_ERR_ARG;
    cudaStream_t st = nullptr;
    int *d_err = nullptr, h = -1;
    G2_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) {
        cudaStreamDestroy(st);
        return G2_ERR_NOMEM;
    }
    cudaMemsetAsync(d_err, 0, sizeof(int), st);
    k_wait_unarrived<<<1, 32, 0, st>>>(d_err, (unsigned long long)limit_ms * 1000000ull);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d_err);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) {
        g2_set_error(__FILE__, __LINE__, cudaGetErrorString(e));
        return G2_ERR_CUDA;
    }
    g2_count_launches(1);
    return h;  // 77 when the wait gave up as designed
}
