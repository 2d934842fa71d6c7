// BF16 GEMM on the 5th-generation tensor cores (tcgen05, accumulators in tensor memory), FP32 output:
//     C[M][N] = A[M][K] * B[N][K]^T   (+ C when accumulate != 0)
// A and B are K-major (row-major with K contiguous), the canonical operand form of tcgen05.mma.  The
// learned preconditioner's 3-D convolutions run on it (forward: im2col x weights; backward: the same
// kernel on transposed operands).
//
// CTA tile 128 x BN, K tile 64, two shared-memory stages.  All 128 threads stage A and B tiles with
// 16-byte cp.async into the SWIZZLE_NONE K-major layout (8-row x 16-byte core matrices: row step 16 B,
// row-group step SBO = 128 B, 8-element K-chunk step LBO = rows*16 B), make them visible to the async
// proxy, and one thread issues four tcgen05.mma (K = 16 each) per tile and commits them to the stage's
// mbarrier.  The epilogue reads the accumulator with tcgen05.ld (warp w reads TMEM lanes 32w..32w+31,
// i.e. rows 32w..) and stores FP32.  Every mbarrier wait is bounded (2 s) and reports through the
// error word.
#include <cstdint>
#include <cuda_bf16.h>
#include "common.cuh"
#include "ie_internal.h"
#include "tma.cuh"

namespace {

constexpr int BM = 128, BK = 64, NTH = 128;

G2_D uint32_t smem_u32(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

G2_D void cp_async16(void *dst, const void *src, bool valid)
{
    const int n = valid ? 16 : 0;  // src-size 0: zero fill
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(n) : "memory");
}

// SWIZZLE_NONE K-major shared-memory matrix descriptor (sm100 version 1)
G2_D uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // version
    // base offset 0, lbo mode 0, layout type 0 (SWIZZLE_NONE)
    return d;
}

// instruction descriptor: BF16 x BF16 -> F32, K-major A and B, M = 128, N = n
__host__ __device__ constexpr uint32_t umma_idesc(int n)
{
    return (1u << 4)                      // D format F32
           | (1u << 7)                    // A format BF16
           | (1u << 10)                   // B format BF16
           | ((uint32_t)(n >> 3) << 17)   // N >> 3
           | ((uint32_t)(BM >> 4) << 24); // M >> 4
}

G2_D void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

G2_D void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// offset of element (r, k) of a rows x 64 K-major tile in the core-matrix layout
G2_D int tile_off(int r, int kc, int rows) { return kc * rows * 16 + (r >> 3) * 128 + (r & 7) * 16; }

template <int BN>
__global__ void __launch_bounds__(NTH, 1) k_gemm_bf16_tn(const __nv_bfloat16 *__restrict__ A,
                                                        const __nv_bfloat16 *__restrict__ B, float *__restrict__ C,
                                                        int M, int N, int K, int lda, int ldb, int ldc,
                                                        int accumulate, int *err)
{
    constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE = A_BYTES + B_BYTES;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * STAGE);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;

    const int nk = (K + BK - 1) / BK;
    bool ok = true;
    for (int kt = 0; kt < nk; kt++) {
        const int s = kt & 1;
        unsigned char *sa = smem + s * STAGE, *sb = sa + A_BYTES;
        if (kt >= 2) ok = ok && mbar_wait_bounded(&bar[s], (uint32_t)(((kt >> 1) - 1) & 1), err, 31);
        const int k0 = kt * BK;
        for (int i = tid; i < BM * 8; i += NTH) {  // A: 128 rows x 8 chunks of 8 elements
            const int r = i >> 3, kc = i & 7, gr = m0 + r, gk = k0 + kc * 8;
            const bool v = gr < M && gk < K;
            cp_async16(sa + tile_off(r, kc, BM), v ? A + (size_t)gr * lda + gk : A, v);
        }
        for (int i = tid; i < BN * 8; i += NTH) {
            const int r = i >> 3, kc = i & 7, gr = n0 + r, gk = k0 + kc * 8;
            const bool v = gr < N && gk < K;
            cp_async16(sb + tile_off(r, kc, BN), v ? B + (size_t)gr * ldb + gk : B, v);
        }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0 && ok) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t ab = smem_u32(sa), bb = smem_u32(sb);
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++) {
                const uint64_t ad = umma_desc(ab + 2 * kk * BM * 16, BM * 16, 128);
                const uint64_t bd = umma_desc(bb + 2 * kk * BN * 16, BN * 16, 128);
                umma_bf16(tmem, ad, bd, umma_idesc(BN), (kt > 0 || kk > 0) ? 1u : 0u);
            }
            umma_commit(&bar[s]);
        }
    }
    // the last commit completes after every earlier MMA of this thread
    ok = ok && mbar_wait_bounded(&bar[(nk - 1) & 1], (uint32_t)(((nk - 1) >> 1) & 1), err, 32);
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + lane_base + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
                float *dst = C + (size_t)row * ldc + n0 + c0;
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    if (n0 + c0 + j < N) {
                        const float x = __uint_as_float(v[j]);
                        dst[j] = accumulate > 0 ? dst[j] + x : x;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

template <int BN>
int launch_gemm(const void *A, const void *B, float *C, int M, int N, int K, int lda, int ldb, int ldc, int acc,
                int *err, cudaStream_t st)
{
    constexpr int SMEM = 2 * (BM * BK * 2 + BN * BK * 2) + 64;
    static bool attr = false;
    if (!attr) {
        G2_CUDA_CHECK(cudaFuncSetAttribute(k_gemm_bf16_tn<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
        attr = true;
    }
    dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN);
    k_gemm_bf16_tn<BN><<<grid, NTH, SMEM, st>>>(reinterpret_cast<const __nv_bfloat16 *>(A),
                                                reinterpret_cast<const __nv_bfloat16 *>(B), C, M, N, K, lda, ldb, ldc,
                                                acc, err);
    G2_CUDA_CHECK(cudaGetLastError());
    return G2_OK;
}

}  // namespace

// C = A B^T (accumulate = 0), C += A B^T (accumulate = 1); K, lda, ldb multiples of 8 (16-byte rows)
int ie_gemm_bf16_tn(const void *A, const void *B, float *C, int M, int N, int K, int lda, int ldb, int ldc,
                    int accumulate, int *err, cudaStream_t st)
{
    if (M <= 0 || N <= 0 || K <= 0 || (K % 8) || (lda % 8) || (ldb % 8) || lda < K || ldb < K || ldc < N)
        return G2_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15) return G2_ERR_ARG;
    if (N <= 32) return launch_gemm<32>(A, B, C, M, N, K, lda, ldb, ldc, accumulate, err, st);
    if (N <= 64) return launch_gemm<64>(A, B, C, M, N, K, lda, ldb, ldc, accumulate, err, st);
    return launch_gemm<128>(A, B, C, M, N, K, lda, ldb, ldc, accumulate, err, st);
}
