// 3x3x3 convolutions of the learned preconditioner as GEMMs on the tcgen05 kernel (umma_gemm.cu).
//
// Activations are channels-last: x[v][c], v = ((n*D + z)*H + y)*W + x_, bf16.  A convolution with
// stride s and padding 1 is Y[v'][co] = sum_k cols[v'][k] Wt[co][k] with k = tap*C + c,
// tap = (dz*3 + dy)*3 + dx, and cols[v'][tap*C + c] = x[(n, z'*s + dz - 1, y'*s + dy - 1, x'*s + dx - 1)][c]
// (zero outside the volume; zero in the padding columns k >= 27C up to Kp, a multiple of 8 so that
// every GEMM row is 16-byte aligned).
//   forward        Y  = cols(x) Wt^T                     (GEMM, then bias-free activation in the caller)
//   weight grad    dW = dY^T cols(x)                      (GEMM on transposed operands)
//   input grad     dcols = dY Wt,  dx = col2im(dcols)     (GEMM, then the gather below)
// col2im is written as a gather (each input voxel sums the taps that read it), so it needs no atomics
// and its summation order is fixed.
#include <cuda_bf16.h>
#include "common.cuh"
#include "ie_internal.h"

namespace {

__global__ void k_im2col3d(const __nv_bfloat16 *__restrict__ x, __nv_bfloat16 *__restrict__ cols, int N, int D,
                           int H, int W, int C, int s, int Do, int Ho, int Wo, int Kp)
{
    const long long total = (long long)N * Do * Ho * Wo * Kp;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i % Kp);
        long long v = i / Kp;
        __nv_bfloat16 val = __float2bfloat16(0.f);
        if (k < 27 * C) {
            const int c = k % C, tap = k / C;
            const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
            const int xo = (int)(v % Wo);
            v /= Wo;
            const int yo = (int)(v % Ho);
            v /= Ho;
            const int zo = (int)(v % Do);
            const int n = (int)(v / Do);
            const int zi = zo * s + dz - 1, yi = yo * s + dy - 1, xi = xo * s + dx - 1;
            if (zi >= 0 && zi < D && yi >= 0 && yi < H && xi >= 0 && xi < W)
                val = x[((((long long)n * D + zi) * H + yi) * W + xi) * C + c];
        }
        cols[i] = val;
    }
}

// C a multiple of 8 (every layer of the network): one thread per 16-byte vector (8 channels) of a cols
// row, 32-bit index arithmetic; consecutive threads write consecutive vectors of a row
__global__ void k_im2col3d_v8(const uint4 *__restrict__ x, uint4 *__restrict__ cols, int D, int H, int W, int C8,
                              int s, int Do, int Ho, int Wo, int Kp8, int total)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int v = i / Kp8, kv = i - v * Kp8;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (kv < 27 * C8) {
            const int tap = kv / C8, q = kv - tap * C8;
            const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
            int r = v;
            const int xo = r % Wo;
            r /= Wo;
            const int yo = r % Ho;
            r /= Ho;
            const int zo = r % Do;
            const int n = r / Do;
            const int zi = zo * s + dz - 1, yi = yo * s + dy - 1, xi = xo * s + dx - 1;
            if (zi >= 0 && zi < D && yi >= 0 && yi < H && xi >= 0 && xi < W)
                val = x[(((long long)(n * D + zi) * H + yi) * W + xi) * C8 + q];
        }
        cols[i] = val;
    }
}

// dx[v][c] = sum over taps of dcols[v'][tap*C + c] for the output voxels v' that read v at that tap
__global__ void k_col2im3d(const float *__restrict__ dcols, float *__restrict__ dx, int N, int D, int H, int W,
                           int C, int s, int Do, int Ho, int Wo, int Kp)
{
    const long long total = (long long)N * D * H * W * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        long long v = i / C;
        const int xi = (int)(v % W);
        v /= W;
        const int yi = (int)(v % H);
        v /= H;
        const int zi = (int)(v % D);
        const int n = (int)(v / D);
        float acc = 0.f;
        for (int dz = 0; dz < 3; dz++) {
            const int tz = zi + 1 - dz;
            if (tz < 0 || tz % s) continue;
            const int zo = tz / s;
            if (zo >= Do) continue;
            for (int dy = 0; dy < 3; dy++) {
                const int ty = yi + 1 - dy;
                if (ty < 0 || ty % s) continue;
                const int yo = ty / s;
                if (yo >= Ho) continue;
                for (int dxx = 0; dxx < 3; dxx++) {
                    const int tx = xi + 1 - dxx;
                    if (tx < 0 || tx % s) continue;
                    const int xo = tx / s;
                    if (xo >= Wo) continue;
                    const long long vo = (((long long)n * Do + zo) * Ho + yo) * Wo + xo;
                    acc += dcols[vo * Kp + ((dz * 3 + dy) * 3 + dxx) * C + c];
                }
            }
        }
        dx[i] = acc;
    }
}

int grid_for(long long n)
{
    long long g = (n + 255) / 256;
    return (int)(g < 148LL * 16 ? g : 148LL * 16);
}

}  // namespace

int ie_im2col3d(const void *x, void *cols, int N, int D, int H, int W, int C, int s, int Kp, cudaStream_t st)
{
    if (N < 1 || D < 1 || H < 1 || W < 1 || C < 1 || (s != 1 && s != 2) || Kp < 27 * C || (Kp % 8)) return G2_ERR_ARG;
    const int Do = (D - 1) / s + 1, Ho = (H - 1) / s + 1, Wo = (W - 1) / s + 1;
    const long long total = (long long)N * Do * Ho * Wo * Kp;
    const long long total8 = total / 8;
    if (C % 8 == 0 && total8 < (1LL << 30) && (reinterpret_cast<uintptr_t>(x) % 16) == 0 &&
        (reinterpret_cast<uintptr_t>(cols) % 16) == 0) {
        k_im2col3d_v8<<<grid_for(total8), 256, 0, st>>>(reinterpret_cast<const uint4 *>(x),
                                                         reinterpret_cast<uint4 *>(cols), D, H, W, C / 8, s, Do, Ho,
                                                         Wo, Kp / 8, (int)total8);
        G2_CUDA_CHECK(cudaGetLastError());
        return G2_OK;
    }
    k_im2col3d<<<grid_for(total), 256, 0, st>>>(reinterpret_cast<const __nv_bfloat16 *>(x),
                                                reinterpret_cast<__nv_bfloat16 *>(cols), N, D, H, W, C, s, Do, Ho, Wo, Kp);
    G2_CUDA_CHECK(cudaGetLastError());
    return G2_OK;
}

int ie_col2im3d(const float *dcols, float *dx, int N, int D, int H, int W, int C, int s, int Kp, cudaStream_t st)
{
    if (N < 1 || D < 1 || H < 1 || W < 1 || C < 1 || (s != 1 && s != 2) || Kp < 27 * C) return G2_ERR_ARG;
    const int Do = (D - 1) / s + 1, Ho = (H - 1) / s + 1, Wo = (W - 1) / s + 1;
    const long long total = (long long)N * D * H * W * C;
    k_col2im3d<<<grid_for(total), 256, 0, st>>>(dcols, dx, N, D, H, W, C, s, Do, Ho, Wo, Kp);
    G2_CUDA_CHECK(cudaGetLastError());
    return G2_OK;
}
