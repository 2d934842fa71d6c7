// Common device helpers: complex arithmetic on double2/float2 and error handling.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#define G2_HD __host__ __device__ __forceinline__
#define G2_D __device__ __forceinline__

template <typename R> struct Cplx;
template <> struct Cplx<double> { using T = double2; };
template <> struct Cplx<float> { using T = float2; };

G2_HD double2 mk(double a, double b) { return make_double2(a, b); }
G2_HD float2 mk(float a, float b) { return make_float2(a, b); }

template <typename C> G2_HD C czero();
template <> G2_HD double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> G2_HD float2 czero<float2>() { return make_float2(0.f, 0.f); }

G2_HD double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
G2_HD double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
G2_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
G2_HD float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
G2_HD double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
G2_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
G2_HD double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
G2_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
G2_HD double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
G2_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// acc += a*b
G2_HD void cfma(double2 &acc, double2 a, double2 b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
G2_HD void cfma(float2 &acc, float2 a, float2 b)
{
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
}
// complex division a/b (Smith's algorithm)
G2_HD double2 cdiv(double2 a, double2 b)
{
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.y + b.x * r;
        return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}

template <typename C> G2_HD C to_c(double2 v);
template <> G2_HD double2 to_c<double2>(double2 v) { return v; }
template <> G2_HD float2 to_c<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }

G2_HD int ilog2(int n)
{
    int l = 0;
    while ((1 << l) < n) l++;
    return l;
}
G2_D int bitrev(int v, int bits) { return (int)(__brev((unsigned)v) >> (32 - bits)); }

// In-place radix-2 DIT FFT of `nlines` lines of length L = 2^log2L held in shared memory.
// Element i of line l lives at s[l*ls + i*es]; the data must already be in bit-reversed order.
// tw[j] = exp(-2*pi*i*j/L) for j < L/2 (forward); inverse uses the conjugates.  Unnormalised.
// LINE_FAST selects the thread->butterfly mapping (line index fastest when lines are interleaved).
template <typename C, bool LINE_FAST>
G2_D void smem_fft(C *s, int log2L, int nlines, int ls, int es, const C *__restrict__ tw, bool inverse)
{
    const int L = 1 << log2L, half = L >> 1;
    const int nb = nlines * half;
    for (int lh = 0; lh < log2L; lh++) {
        const int h = 1 << lh;
        const int tshift = log2L - 1 - lh;  // twiddle index j * (L/(2h))
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            int line, k;
            if (LINE_FAST) { line = b % nlines; k = b / nlines; }
            else { k = b & (half - 1); line = b >> (log2L - 1); }
            const int j = k & (h - 1);
            const int i0 = ((k >> lh) << (lh + 1)) + j;
            C w = tw[j << tshift];
            if (inverse) w.y = -w.y;
            C *p0 = s + line * ls + i0 * es;
            C *p1 = p0 + h * es;
            C a = *p0, bb = cmul(*p1, w);
            *p0 = a + bb;
            *p1 = a - bb;
        }
        __syncthreads();
    }
}

// Device layout of the full (xz, yz) Nz x Nz blocks: column-major with the row index XOR-swizzled by
// the low bits of the column, so lane-parallel reads of a row and of a column both hit distinct
// shared-memory banks.  W = 1 is plain column-major.
G2_HD int asw(int r, int c, int N, int W) { return c * N + (r ^ (c & (W - 1))); }
// swizzle widths used for the FP64 and FP32 device tensors
__host__ __device__ constexpr int asw_width64(int Nz) { return (Nz % 8 == 0) ? 8 : 1; }
__host__ __device__ constexpr int asw_width32(int Nz) { return (Nz % 16 == 0) ? 16 : ((Nz % 8 == 0) ? 8 : 1); }

#define G2_CUDA_CHECK(expr)                                                                    \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            g2_set_error(__FILE__, __LINE__, cudaGetErrorString(e_));                          \
            return G2_ERR_CUDA;                                                                \
        }                                                                                      \
    } while (0)

void g2_set_error(const char *file, int line, const char *msg);
