// Four-step FFT of many short lines inside one CTA: register DFTs + one shared-memory transpose.
//
// A line of length L = N1*N2 (power of two) is transformed as
//   step 1: thread (line, n1) loads x[n1 + N1*n2], n2 < N2, does an N2-point DFT in registers,
//           multiplies by W_L^(n1*k2) and parks the N2 values in shared memory;
//   step 2: thread (line, k2) reads the N1 values of column k2, does an N1-point DFT in registers,
//           and emits X[k2 + N2*k1].
// PAD_IN: inputs with index >= L/2 are zero (zero-padded transform) and are neither loaded nor
// multiplied.  CROP_OUT: only outputs with index < L/2 are produced.
// Register DFTs are radix-2 decimation-in-frequency with compile-time indexing; the twiddles come from
// one table tw[j] = exp(-2 pi i j / L), j < L, held in shared memory, except the factors -i (+i in the
// inverse), which the register DFTs apply exactly as a swap and a sign (7 of the 17 twiddle products of a
// 16-point DFT).
#pragma once
#include "common.cuh"

template <int N> struct Log2 { static constexpr int v = 1 + Log2<N / 2>::v; };
template <> struct Log2<1> { static constexpr int v = 0; };

__host__ __device__ constexpr int brev_c(int v, int bits)
{
    int r = 0;
    for (int i = 0; i < bits; i++) r |= ((v >> i) & 1) << (bits - 1 - i);
    return r;
}

template <typename C, bool INV>
G2_D C twid(const C *tw, int idx)
{
    C w = tw[idx];
    if (INV) w.y = -w.y;
    return w;
}

// d * W_N^e for the register DFTs: e = 0 is 1 and e = N/4 is -i (forward) or +i (inverse), exactly (a
// swap and a sign); other exponents read the table.
template <typename C, int N, bool INV>
G2_D C twiddle_mul(C d, int e, const C *tw, int Lstride)
{
    if (e == 0) return d;
    if (4 * e == N) {
        C r;
        if (INV) { r.x = -d.y; r.y = d.x; }
        else { r.x = d.y; r.y = -d.x; }
        return r;
    }
    return cmul(d, twid<C, INV>(tw, e * Lstride));
}

// Butterfly sum and difference.  Complex64 uses one packed add.rn.f32x2 / sub.rn.f32x2 (sm_100) each, which
// round like two scalar adds: the register DFTs issue half the add instructions (the y passes are
// issue-bound).
G2_D double2 bf_add(double2 a, double2 b) { return a + b; }
G2_D double2 bf_sub(double2 a, double2 b) { return a - b; }
G2_D float2 bf_add(float2 a, float2 b)
{
    union U { float2 f; unsigned long long u; } ua, ub, uc;
    ua.f = a;
    ub.f = b;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(uc.u) : "l"(ua.u), "l"(ub.u));
    return uc.f;
}
G2_D float2 bf_sub(float2 a, float2 b)
{
    union U { float2 f; unsigned long long u; } ua, ub, uc;
    ua.f = a;
    ub.f = b;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(uc.u) : "l"(ua.u), "l"(ub.u));
    return uc.f;
}

// In-place N-point DFT of a[] (natural order in, bit-reversed order out).  L/N is the table stride.
// If HALF_ZERO, a[N/2..N-1] are zero on entry (first stage pruned).
template <typename C, int N, bool INV, bool HALF_ZERO>
G2_D void reg_dft_dif(C (&a)[N], const C *tw, int Lstride)
{
#pragma unroll
    for (int h = N / 2; h >= 1; h /= 2) {
#pragma unroll
        for (int g = 0; g < N; g += 2 * h) {
#pragma unroll
            for (int j = 0; j < h; j++) {
                const C u = a[g + j];
                if (HALF_ZERO && h == N / 2) {
                    a[g + j] = u;
                    a[g + j + h] = twiddle_mul<C, N, INV>(u, j * (N / (2 * h)), tw, Lstride);
                } else {
                    const C v = a[g + j + h];
                    a[g + j] = bf_add(u, v);
                    a[g + j + h] = twiddle_mul<C, N, INV>(bf_sub(u, v), j * (N / (2 * h)), tw, Lstride);
                }
            }
        }
    }
}

// One CTA transforms `nl` lines (nl <= 2^lg_nl, the CTA's line block).  Functors:
//   load(line, idx) -> C            (step 1 input)
//   store(line, idx, C)             (step 2 output)
//   off(line, n1, k2) -> int        (shared-memory slot of the intermediate)
// LF1/LF2: item ordering (true: line index fastest across threads; false: n1 / k2 fastest).  Items are
// split with shifts and masks of the power-of-two line block; lines >= nl (a partial last block) are
// skipped.  n1 and k2 are masked to their ranges, which changes no value but lets the compiler resolve the
// index arithmetic of the unrolled outputs (a slot mapping per output, for instance) at compile time.
// The same transform run by a subset of the CTA's threads: thread tid of nthr, with sync() the barrier
// of those threads (a named barrier when other warps of the CTA do other work).
template <typename C, int N1, int N2, bool INV, bool PAD_IN, bool CROP_OUT, bool LF1, bool LF2, class LoadF,
          class StoreF, class OffF, class SyncF>
G2_D void fft4step_part(C *sm, int nl, int lg_nl, const C *tw, LoadF load, StoreF store, OffF off, int tid, int nthr,
                        SyncF sync)
{
    constexpr int L = N1 * N2;
    const int nlb = 1 << lg_nl;
    const int n_items1 = (LF1 ? nlb : nl) * N1;
    for (int it = tid; it < n_items1; it += nthr) {
        int line, n1;
        if (LF1) { line = it & (nlb - 1); n1 = (it >> lg_nl) & (N1 - 1); }
        else { n1 = it % N1; line = it / N1; }
        if (LF1 && line >= nl) continue;
        C a[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; n2++) {
            if (PAD_IN && n2 >= N2 / 2) a[n2] = czero<C>();
            else a[n2] = load(line, n1 + N1 * n2);
        }
        reg_dft_dif<C, N2, INV, PAD_IN>(a, tw, L / N2);
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) {
            C v = a[brev_c(k2, Log2<N2>::v)];
            if (k2 != 0 && n1 != 0) v = cmul(v, twid<C, INV>(tw, n1 * k2));
            sm[off(line, n1, k2)] = v;
        }
    }
    sync();
    const int n_items2 = (LF2 ? nlb : nl) * N2;
    for (int it = tid; it < n_items2; it += nthr) {
        int line, k2;
        if (LF2) { line = it & (nlb - 1); k2 = (it >> lg_nl) & (N2 - 1); }
        else { k2 = it % N2; line = it / N2; }
        if (LF2 && line >= nl) continue;
        C a[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) a[n1] = sm[off(line, n1, k2)];
        reg_dft_dif<C, N1, INV, false>(a, tw, L / N1);
#pragma unroll
        for (int k1 = 0; k1 < (CROP_OUT ? N1 / 2 : N1); k1++) store(line, k2 + N2 * k1, a[brev_c(k1, Log2<N1>::v)]);
    }
}

// fft4step_part for a fixed number of step-1 items per thread (IPT * nthr >= the items): every thread issues
// the loads of all its items before the first register DFT, so the transform waits for one load round trip
// instead of one per item (for a few warps that transform tasks one after another).
template <typename C, int N1, int N2, int IPT, bool INV, bool PAD_IN, bool CROP_OUT, class LoadF, class StoreF,
          class OffF, class SyncF>
G2_D void fft4step_part_ilp(C *sm, int nl, int lg_nl, const C *tw, LoadF load, StoreF store, OffF off, int tid,
                            int nthr, SyncF sync)
{
    constexpr int L = N1 * N2;
    constexpr int NLD = PAD_IN ? N2 / 2 : N2;
    const int nlb = 1 << lg_nl;
    const int n_items1 = nlb * N1;  // line index fastest
    C a[IPT][N2];
#pragma unroll
    for (int r = 0; r < IPT; r++) {
        const int it = tid + r * nthr;
        const int line = it & (nlb - 1), n1 = (it >> lg_nl) & (N1 - 1);
        const bool ok = it < n_items1 && line < nl;
#pragma unroll
        for (int n2 = 0; n2 < N2; n2++) a[r][n2] = (ok && n2 < NLD) ? load(line, n1 + N1 * n2) : czero<C>();
    }
#pragma unroll
    for (int r = 0; r < IPT; r++) {
        const int it = tid + r * nthr;
        const int line = it & (nlb - 1), n1 = (it >> lg_nl) & (N1 - 1);
        if (it >= n_items1 || line >= nl) continue;
        reg_dft_dif<C, N2, INV, PAD_IN>(a[r], tw, L / N2);
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) {
            C v = a[r][brev_c(k2, Log2<N2>::v)];
            if (k2 != 0 && n1 != 0) v = cmul(v, twid<C, INV>(tw, n1 * k2));
            sm[off(line, n1, k2)] = v;
        }
    }
    sync();
    const int n_items2 = nlb * N2;
    for (int it = tid; it < n_items2; it += nthr) {
        const int line = it & (nlb - 1), k2 = (it >> lg_nl) & (N2 - 1);
        if (line >= nl) continue;
        C b[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) b[n1] = sm[off(line, n1, k2)];
        reg_dft_dif<C, N1, INV, false>(b, tw, L / N1);
#pragma unroll
        for (int k1 = 0; k1 < (CROP_OUT ? N1 / 2 : N1); k1++) store(line, k2 + N2 * k1, b[brev_c(k1, Log2<N1>::v)]);
    }
}

// fft4step for a store that needs other data at each output (an epilogue): pre(line, idx) returns it and is
// called for all of an item's outputs before the item's shared-memory loads and register DFT, so those global
// loads are in flight together (a store functor that loads would otherwise wait once per output: the
// compiler may not move a load above an earlier store to possibly aliasing memory); store(line, idx, v, p).
// Each output's data is read before that thread stores any output, so in-place vectors stay correct.
template <typename C, int N1, int N2, bool INV, bool PAD_IN, bool CROP_OUT, bool LF1, bool LF2, class LoadF,
          class PreF, class StoreF, class OffF>
G2_D void fft4step_pre(C *sm, int nl, int lg_nl, const C *tw, LoadF load, PreF pre, StoreF store, OffF off)
{
    constexpr int L = N1 * N2;
    constexpr int NOUT = CROP_OUT ? N1 / 2 : N1;
    const int nlb = 1 << lg_nl;
    const int n_items1 = (LF1 ? nlb : nl) * N1;
    for (int it = threadIdx.x; it < n_items1; it += blockDim.x) {
        int line, n1;
        if (LF1) { line = it & (nlb - 1); n1 = (it >> lg_nl) & (N1 - 1); }
        else { n1 = it % N1; line = it / N1; }
        if (LF1 && line >= nl) continue;
        C a[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; n2++) {
            if (PAD_IN && n2 >= N2 / 2) a[n2] = czero<C>();
            else a[n2] = load(line, n1 + N1 * n2);
        }
        reg_dft_dif<C, N2, INV, PAD_IN>(a, tw, L / N2);
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) {
            C v = a[brev_c(k2, Log2<N2>::v)];
            if (k2 != 0 && n1 != 0) v = cmul(v, twid<C, INV>(tw, n1 * k2));
            sm[off(line, n1, k2)] = v;
        }
    }
    __syncthreads();
    const int n_items2 = (LF2 ? nlb : nl) * N2;
    for (int it = threadIdx.x; it < n_items2; it += blockDim.x) {
        int line, k2;
        if (LF2) { line = it & (nlb - 1); k2 = (it >> lg_nl) & (N2 - 1); }
        else { k2 = it % N2; line = it / N2; }
        if (LF2 && line >= nl) continue;
        decltype(pre(0, 0)) p[NOUT];
#pragma unroll
        for (int k1 = 0; k1 < NOUT; k1++) p[k1] = pre(line, k2 + N2 * k1);
        C a[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) a[n1] = sm[off(line, n1, k2)];
        reg_dft_dif<C, N1, INV, false>(a, tw, L / N1);
#pragma unroll
        for (int k1 = 0; k1 < NOUT; k1++) store(line, k2 + N2 * k1, a[brev_c(k1, Log2<N1>::v)], p[k1]);
    }
}

// The whole CTA transforms its line block.
template <typename C, int N1, int N2, bool INV, bool PAD_IN, bool CROP_OUT, bool LF1, bool LF2, class LoadF,
          class StoreF, class OffF>
G2_D void fft4step(C *sm, int nl, int lg_nl, const C *tw, LoadF load, StoreF store, OffF off)
{
    fft4step_part<C, N1, N2, INV, PAD_IN, CROP_OUT, LF1, LF2>(sm, nl, lg_nl, tw, load, store, off, (int)threadIdx.x,
                                                              (int)blockDim.x, [] { __syncthreads(); });
}

// factorisation L = N1 * N2 used by the transform kernels
template <int L> struct Fact;
template <> struct Fact<4> { static constexpr int N1 = 2, N2 = 2; };
template <> struct Fact<8> { static constexpr int N1 = 4, N2 = 2; };
template <> struct Fact<16> { static constexpr int N1 = 4, N2 = 4; };
template <> struct Fact<32> { static constexpr int N1 = 8, N2 = 4; };
template <> struct Fact<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct Fact<128> { static constexpr int N1 = 16, N2 = 8; };
template <> struct Fact<256> { static constexpr int N1 = 16, N2 = 16; };
template <> struct Fact<512> { static constexpr int N1 = 32, N2 = 16; };
template <> struct Fact<1024> { static constexpr int N1 = 32, N2 = 32; };
