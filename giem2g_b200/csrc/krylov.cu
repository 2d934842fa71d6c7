// Nested flexible GMRES on the GPU: GFGMRES (GFGMRES/gmres.F90, seq_fgmres.F90) as used by
// GIEM2G_FGMRES (ie_solver_module.F90:141-258), depth 2.
//
//   outer: flexible GMRES, FP64 (complex128) basis, Hessenberg, Givens and true residual;
//          right preconditioner = one cycle of the inner GMRES (FGMRES_BASED_PRECONDITIONER).
//   inner: GMRES, MaxIt = 1, x0 = b = v_in, complex128 (plain mode) or complex64 (mixed mode).
//
// Arnoldi uses the reference's iterated classical Gram-Schmidt (gmres.F90:263-281): up to four
// passes, stop when 2||w|| > ||h_pass||; each pass after the first is ONE sweep over the basis that
// subtracts V h, and accumulates the next pass's dots and ||w||^2.  Complex Givens rotations follow
// the netlib ZROTG/ZROT definitions; restarts use the Arnoldi residual (RESTART_RESIDUAL = .FALSE.).
// Dot products accumulate in FP64 for both precisions.
//
// The inner solve is a fixed launch sequence whose kernels are gated by device flags, so it needs no
// host round trip; the outer loop reads two scalars back once per outer iteration (Inform callback).
// The inner solver's closing true-residual apply (gmres.F90:403) produces a number nobody reads; it
// is skipped unless the environment variable GIEM2G_INNER_TRUE_RESIDUAL=1 asks for it (the solution
// and iteration history are the same either way; only the apply count differs).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>
#include "common.cuh"
#include "krylov.h"

namespace {

constexpr int kVT = 256;   // threads of the vector kernels
constexpr int kILP = 4;    // elements per thread and iteration of the element-wise vector kernels
constexpr int KMAX = 32;   // largest basis handled in one sweep
constexpr double ZERO_THRESHOLD = 1e-14;  // gmres.F90:21
constexpr int N_IGS = 3;                  // gmres.F90:22
constexpr double kHookGain = 0.5;         // an outer step through the hook must halve the misfit

enum { F_KRYLOV = 0, F_PASS = 1, F_L = 2, F_ITER = 3, F_SOLVER = 4, F_NFLAGS = 8 };
enum { S_BN = 0, S_BETA = 1, S_DNORMW = 2, S_DLOO = 3, S_BEA = 4, S_NRM2 = 5, S_NSCAL = 8 };

struct Level {
    int m = 0;
    double2 *H = nullptr;   // (m+1) x (m+1) column-major, column m holds g
    double *cs = nullptr;
    double2 *sn = nullptr;
    double2 *hpass = nullptr, *hnext = nullptr, *y = nullptr;
    double *scal = nullptr;
    int *flags = nullptr;
    unsigned *counter = nullptr;  // blocks done, for the last-block reductions (back to 0 after each use)
};

G2_HD int hix(int i, int j, int m) { return i + j * (m + 1); }

template <typename C> G2_D double2 ld2(const C *p, size_t i);
template <> G2_D double2 ld2<double2>(const double2 *p, size_t i) { return p[i]; }
template <> G2_D double2 ld2<float2>(const float2 *p, size_t i)
{
    const float2 v = p[i];
    return make_double2(v.x, v.y);
}
template <typename C> G2_D void st2(C *p, size_t i, double2 v);
template <> G2_D void st2<double2>(double2 *p, size_t i, double2 v) { p[i] = v; }
template <> G2_D void st2<float2>(float2 *p, size_t i, double2 v) { p[i] = make_float2((float)v.x, (float)v.y); }

// The basis sweeps move 16-byte words: two complex64 values per load (complex128 values are 16 bytes
// already).  On a B200 a two-instance sweep of 11 complex64 vectors of 1.57 M elements took 84 us with
// 8-byte loads and 52 us with 16-byte loads.  Vectors whose length (and column stride) is odd keep
// element-wise loads, since their odd columns are not 16-byte aligned.
template <typename C> struct Wide;
template <> struct Wide<float2> {
    using T = float4;
    static constexpr int E = 2;
};
template <> struct Wide<double2> {
    using T = double2;
    static constexpr int E = 1;
};
G2_D float2 part_of(const float4 &p, int e) { return e ? make_float2(p.z, p.w) : make_float2(p.x, p.y); }
G2_D double2 part_of(const double2 &p, int) { return p; }
G2_D void set_part(float4 &p, int e, float2 v)
{
    if (e) {
        p.z = v.x;
        p.w = v.y;
    } else {
        p.x = v.x;
        p.y = v.y;
    }
}
G2_D void set_part(double2 &p, int, double2 v) { p = v; }
// words of E elements over the whole vector, or 0 when the lengths do not allow them
template <typename C> G2_D size_t wide_words(size_t N, size_t ld)
{
    constexpr int E = Wide<C>::E;
    return (N % E == 0 && ld % E == 0) ? N / E : 0;
}

template <typename C> struct RealOf;
template <> struct RealOf<double2> { using T = double; };
template <> struct RealOf<float2> { using T = float; };

// per-thread partial sums in the vector's precision (a handful of elements each), block and grid
// reductions in FP64
template <int KM, typename R>
G2_D void block_reduce_store_r(R (&ax)[KM + 1], R (&ay)[KM + 1], double2 *part)
{
    __shared__ double2 red[kVT / 32][KM + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k <= KM; k++) {
        double vx = ax[k], vy = ay[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            vx += __shfl_xor_sync(0xffffffffu, vx, o);
            vy += __shfl_xor_sync(0xffffffffu, vy, o);
        }
        if (lane == 0) red[warp][k] = make_double2(vx, vy);
    }
    __syncthreads();
    if (threadIdx.x <= KM) {
        double2 s = make_double2(0.0, 0.0);
        for (int w = 0; w < kVT / 32; w++) {
            s.x += red[w][threadIdx.x].x;
            s.y += red[w][threadIdx.x].y;
        }
        part[(size_t)blockIdx.x * (KMAX + 1) + (threadIdx.x == KM ? KMAX : threadIdx.x)] = s;
    }
}

// ---- scalar control kernels (one thread) -------------------------------------------------------
// first CGS pass of step j: H(0..j, j) = h, hpass = h, pass active
G2_D void cgs_first_body(Level &L, int j, const double2 *h)
{
    for (int i = 0; i <= j; i++) {
        L.H[hix(i, j, L.m)] = h[i];
        L.hpass[i] = h[i];
    }
    L.flags[F_PASS] = 1;
}
// after pass p (1-based) subtracted hpass: decide on another pass (gmres.F90:277-280)
G2_D void cgs_next_body(Level &L, int j, int p)
{
    double dl = 0.0;
    for (int i = 0; i <= j; i++) dl += L.hpass[i].x * L.hpass[i].x + L.hpass[i].y * L.hpass[i].y;
    const double dloo = sqrt(dl), dnormw = sqrt(L.scal[S_NRM2]);
    L.scal[S_DLOO] = dloo;
    L.scal[S_DNORMW] = dnormw;
    if (2.0 * dnormw > dloo || p > N_IGS) {
        L.flags[F_PASS] = 0;
    } else {
        for (int i = 0; i <= j; i++) {
            L.H[hix(i, j, L.m)].x += L.hnext[i].x;
            L.H[hix(i, j, L.m)].y += L.hnext[i].y;
            L.hpass[i] = L.hnext[i];
        }
    }
}

G2_D double cabs_(double2 a) { return hypot(a.x, a.y); }
G2_D double2 cmul_(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
G2_D double2 cdivr(double2 a, double r) { return make_double2(a.x / r, a.y / r); }
// netlib ZROT on one pair
G2_D void zrot1(double2 &cx, double2 &cy, double c, double2 s)
{
    const double2 t = make_double2(c * cx.x + (s.x * cy.x - s.y * cy.y), c * cx.y + (s.x * cy.y + s.y * cy.x));
    const double2 sc = make_double2(s.x, -s.y);
    cy = make_double2(c * cy.x - (sc.x * cx.x - sc.y * cx.y), c * cy.y - (sc.x * cx.y + sc.y * cx.x));
    cx = t;
}
// netlib ZROTG
G2_D void zrotg(double2 &ca, double2 cb, double &c, double2 &s)
{
    const double aca = cabs_(ca);
    if (aca == 0.0) {
        c = 0.0;
        s = make_double2(1.0, 0.0);
        ca = cb;
    } else {
        const double scale = aca + cabs_(cb);
        const double a1 = cabs_(cdivr(ca, scale)), b1 = cabs_(cdivr(cb, scale));
        const double norm = scale * sqrt(a1 * a1 + b1 * b1);
        const double2 alpha = cdivr(ca, aca);
        c = aca / norm;
        s = cdivr(cmul_(alpha, make_double2(cb.x, -cb.y)), norm);
        ca = make_double2(alpha.x * norm, alpha.y * norm);
    }
}

// end of Arnoldi step j (gmres.F90:283-326): H(j+1,j), rotations, Arnoldi misfit, exit test
G2_D void arnoldi_finish_body(Level &L, int j, double tol)
{
    // run by every thread of one block: column j of H, the rotations so far and g(j), g(j+1) are staged in
    // shared memory with one round of loads; thread 0 then applies the same operations in the same order
    // as a single thread on global memory would (a chain of dependent L2 loads otherwise)
    __shared__ double2 hc[KMAX + 1], sn_s[KMAX], gs[2];
    __shared__ double cs_s[KMAX];
    const int m = L.m;
    for (int i = threadIdx.x; i <= j + 1; i += blockDim.x) hc[i] = L.H[hix(i, j, m)];
    for (int i = threadIdx.x; i < j; i += blockDim.x) {
        cs_s[i] = L.cs[i];
        sn_s[i] = L.sn[i];
    }
    if (threadIdx.x < 2) gs[threadIdx.x] = L.H[hix(j + threadIdx.x, m, m)];
    __syncthreads();
    if (threadIdx.x == 0) {
        const double dnormw = L.scal[S_DNORMW], bn = L.scal[S_BN];
        hc[j + 1] = make_double2(dnormw, 0.0);
        for (int i = 0; i < j; i++) zrot1(hc[i], hc[i + 1], cs_s[i], sn_s[i]);
        double2 h1 = hc[j], sn;
        double c;
        zrotg(h1, hc[j + 1], c, sn);
        zrot1(gs[0], gs[1], c, sn);
        zrot1(hc[j], hc[j + 1], c, sn);
        hc[j + 1] = make_double2(0.0, 0.0);
        L.cs[j] = c;
        L.sn[j] = sn;
        L.H[hix(j, m, m)] = gs[0];
        L.H[hix(j + 1, m, m)] = gs[1];
        const double bea = cabs_(gs[1]) / bn;
        L.scal[S_BEA] = bea;
        L.flags[F_ITER] += 1;
        L.flags[F_L] = j + 1;
        if (bea < tol || j + 1 >= m) L.flags[F_KRYLOV] = 0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= j + 1; i += blockDim.x) L.H[hix(i, j, m)] = hc[i];
}

// ---- fused reductions: the last block to finish sums every block's partials ----------------------
// Each block stores its partials, then counts itself done; the block that counts last reduces all
// partials in a fixed order (lane-strided sums, shuffle tree: the result does not depend on which block
// is last) and runs the scalar step that used to be a separate one-thread launch.  It resets the counter
// for the next use.  Blocks test their gates before any of them can reach the last block, so a flag the
// last block changes cannot be seen half-way through the grid.
G2_D bool last_block(unsigned *counter)
{
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (am_last && threadIdx.x == 0) *counter = 0u;
    return am_last;
}
// sums of part[b][col] over blocks for columns 0..K-1 into h[], and of column KMAX into *nrm (one block)
G2_D void reduce_partials(const double2 *part, int nb, int K, double2 *h, double *nrm)
{
    __threadfence();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = warp; k <= K; k += nw) {
        const int col = (k == K) ? KMAX : k;
        double sx = 0.0, sy = 0.0;
        // eight independent loads per lane and round (rows past nb predicated off): the partials come from
        // L2, and each round is one L2 round trip, so 256 rows cost one
        for (int b0 = 0; b0 < nb; b0 += 256) {
            double2 v[8];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                const int b = b0 + lane + 32 * q;
                v[q] = b < nb ? __ldcg(part + (size_t)b * (KMAX + 1) + col) : make_double2(0.0, 0.0);
            }
            sx += ((v[0].x + v[1].x) + (v[2].x + v[3].x)) + ((v[4].x + v[5].x) + (v[6].x + v[7].x));
            sy += ((v[0].y + v[1].y) + (v[2].y + v[3].y)) + ((v[4].y + v[5].y) + (v[6].y + v[7].y));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
        if (lane == 0) {
            if (k < K) h[k] = make_double2(sx, sy);
            else if (nrm) *nrm = sx;
        }
    }
    __syncthreads();
}

// first CGS pass of Arnoldi step j = K-1: h = V^H w, then H(0..j, j) = h, hpass = h
// elements per thread and round of the basis sweeps: all (K + 1) * U loads of a round are issued before the
// first product, so a round costs one memory round trip; the values held stay within 256 bytes per thread
// (32 complex64 or 16 complex128).  0: the basis is too wide to hold, the sweep loads one element at a time.
template <int K, typename C> struct SweepU {
    static constexpr int B = (K + 1) * (int)sizeof(C);
    static constexpr int v = B * 4 <= 256 ? 4 : (B * 2 <= 256 ? 2 : (B <= 256 ? 1 : 0));
};

template <typename C, int K>
G2_D void dots_first_body(const C *__restrict__ V, size_t ld, const C *__restrict__ w, size_t N, double2 *part,
                          Level &L)
{
    using R = typename RealOf<C>::T;
    using W = typename Wide<C>::T;
    constexpr int E = Wide<C>::E;
    constexpr int U = SweepU<K, W>::v > 0 ? SweepU<K, W>::v : 1;
    R ax[K + 1], ay[K + 1];
#pragma unroll
    for (int k = 0; k <= K; k++) ax[k] = ay[k] = R(0);
    const size_t S = (size_t)gridDim.x * kVT, t0 = blockIdx.x * (size_t)kVT + threadIdx.x;
    const size_t Nw = wide_words<C>(N, ld), ldw = ld / E;
    const W *__restrict__ Vw = reinterpret_cast<const W *>(V);
    const W *__restrict__ ww = reinterpret_cast<const W *>(w);
    size_t i = t0;
    for (; SweepU<K, W>::v > 0 && i + (U - 1) * S < Nw; i += U * S) {
        W wv[U], v[K > 0 ? K : 1][U];
#pragma unroll
        for (int u = 0; u < U; u++) wv[u] = ww[i + u * S];
#pragma unroll
        for (int k = 0; k < K; k++)
#pragma unroll
            for (int u = 0; u < U; u++) v[k][u] = Vw[(size_t)k * ldw + i + u * S];
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int e = 0; e < E; e++) {
                const C a = part_of(wv[u], e);
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const C b = part_of(v[k][u], e);
                    ax[k] += b.x * a.x + b.y * a.y;
                    ay[k] += b.x * a.y - b.y * a.x;
                }
            }
    }
    for (; i < Nw; i += S) {
        const W wv = ww[i];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const W v = Vw[(size_t)k * ldw + i];
#pragma unroll
            for (int e = 0; e < E; e++) {
                const C a = part_of(wv, e), b = part_of(v, e);
                ax[k] += b.x * a.x + b.y * a.y;
                ay[k] += b.x * a.y - b.y * a.x;
            }
        }
    }
    for (i = Nw * E + t0; i < N; i += S) {
        const C wv = w[i];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const C v = V[(size_t)k * ld + i];
            ax[k] += v.x * wv.x + v.y * wv.y;
            ay[k] += v.x * wv.y - v.y * wv.x;
        }
    }
    block_reduce_store_r<K, R>(ax, ay, part);
    if (!last_block(L.counter)) return;
    __shared__ double2 hs[KMAX + 1];
    reduce_partials(part, gridDim.x, K, hs, nullptr);
    if (threadIdx.x == 0) cgs_first_body(L, K - 1, hs);
}
template <typename C, int K>
__global__ void __launch_bounds__(kVT) k_dots_first_t(const C *__restrict__ V, size_t ld, const C *__restrict__ w,
                                                      size_t N, double2 *part, Level L, const int *gate)
{
    if (gate && *gate == 0) return;
    dots_first_body<C, K>(V, ld, w, N, part, L);
}

// Several instances of one batch in one launch (blockIdx.y = instance): the same blocks, partials,
// counters and last-block steps per instance as separate launches, so the results are the same; what
// goes is the launch per instance and its ramp and tail.
constexpr int KMI = 4;
template <typename C>
struct Multi {
    C *V[KMI];
    C *w[KMI];
    double2 *part[KMI];
    Level L[KMI];
    const int *gate[KMI];
};
template <typename C, int K>
__global__ void __launch_bounds__(kVT) k_dots_first_m(Multi<C> mm, size_t ld, size_t N)
{
    const int y = blockIdx.y;
    if (mm.gate[y] && *mm.gate[y] == 0) return;
    Level L = mm.L[y];
    dots_first_body<C, K>(mm.V[y], ld, mm.w[y], N, mm.part[y], L);
}

// CGS pass p of step j = K-1: w -= V hpass; dots of the new w; then the pass decision (gmres.F90:277-280)
template <typename C, int K>
G2_D void cgs_pass_body(const C *__restrict__ V, size_t ld, C *__restrict__ w, size_t N, double2 *part, Level &L,
                        int p)
{
    using R = typename RealOf<C>::T;
    using W = typename Wide<C>::T;
    constexpr int E = Wide<C>::E;
    constexpr int KA = K > 0 ? K : 1;
    __shared__ double2 hsh[KA];
    if (threadIdx.x < K) hsh[threadIdx.x] = L.hpass[threadIdx.x];
    __syncthreads();
    R ax[K + 1], ay[K + 1];
#pragma unroll
    for (int k = 0; k <= K; k++) ax[k] = ay[k] = R(0);
    constexpr int U = SweepU<K, W>::v > 0 ? SweepU<K, W>::v : 1;
    const size_t S = (size_t)gridDim.x * kVT, t0 = blockIdx.x * (size_t)kVT + threadIdx.x;
    const size_t Nw = wide_words<C>(N, ld), ldw = ld / E;
    const W *__restrict__ Vw = reinterpret_cast<const W *>(V);
    W *__restrict__ ww = reinterpret_cast<W *>(w);
    // one element: w -= V hpass, then |w|^2 and the dots of the new w (the basis values stay in registers)
    auto element = [&](C &a, const C *b) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            const R hx = (R)hsh[k].x, hy = (R)hsh[k].y;
            a.x -= b[k].x * hx - b[k].y * hy;
            a.y -= b[k].x * hy + b[k].y * hx;
        }
        ax[K] += a.x * a.x + a.y * a.y;
#pragma unroll
        for (int k = 0; k < K; k++) {
            ax[k] += b[k].x * a.x + b[k].y * a.y;
            ay[k] += b[k].x * a.y - b[k].y * a.x;
        }
    };
    size_t i = t0;
    // U words per round, every load of the round first
    for (; SweepU<K, W>::v > 0 && i + (U - 1) * S < Nw; i += U * S) {
        W wv[U], v[K > 0 ? K : 1][U];
#pragma unroll
        for (int u = 0; u < U; u++) wv[u] = ww[i + u * S];
#pragma unroll
        for (int k = 0; k < K; k++)
#pragma unroll
            for (int u = 0; u < U; u++) v[k][u] = Vw[(size_t)k * ldw + i + u * S];
#pragma unroll
        for (int u = 0; u < U; u++) {
#pragma unroll
            for (int e = 0; e < E; e++) {
                C a = part_of(wv[u], e), b[K > 0 ? K : 1];
#pragma unroll
                for (int k = 0; k < K; k++) b[k] = part_of(v[k][u], e);
                element(a, b);
                set_part(wv[u], e, a);
            }
            ww[i + u * S] = wv[u];
        }
    }
    // the rest (all of it when the basis is too wide to hold): one word at a time, the basis read twice
    for (; i < Nw; i += S) {
        W wv = ww[i];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const W v = Vw[(size_t)k * ldw + i];
            const R hx = (R)hsh[k].x, hy = (R)hsh[k].y;
#pragma unroll
            for (int e = 0; e < E; e++) {
                C a = part_of(wv, e);
                const C b = part_of(v, e);
                a.x -= b.x * hx - b.y * hy;
                a.y -= b.x * hy + b.y * hx;
                set_part(wv, e, a);
            }
        }
        ww[i] = wv;
#pragma unroll
        for (int e = 0; e < E; e++) {
            const C a = part_of(wv, e);
            ax[K] += a.x * a.x + a.y * a.y;
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            const W v = Vw[(size_t)k * ldw + i];
#pragma unroll
            for (int e = 0; e < E; e++) {
                const C a = part_of(wv, e), b = part_of(v, e);
                ax[k] += b.x * a.x + b.y * a.y;
                ay[k] += b.x * a.y - b.y * a.x;
            }
        }
    }
    for (i = Nw * E + t0; i < N; i += S) {
        C wv = w[i];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const C v = V[(size_t)k * ld + i];
            const R hx = (R)hsh[k].x, hy = (R)hsh[k].y;
            wv.x -= v.x * hx - v.y * hy;
            wv.y -= v.x * hy + v.y * hx;
        }
        w[i] = wv;
        ax[K] += wv.x * wv.x + wv.y * wv.y;
#pragma unroll
        for (int k = 0; k < K; k++) {
            const C v = V[(size_t)k * ld + i];
            ax[k] += v.x * wv.x + v.y * wv.y;
            ay[k] += v.x * wv.y - v.y * wv.x;
        }
    }
    block_reduce_store_r<K, R>(ax, ay, part);
    if (!last_block(L.counter)) return;
    __shared__ double2 hs[KMAX + 1];
    __shared__ double nrm;
    reduce_partials(part, gridDim.x, K, hs, &nrm);
    if (threadIdx.x < K) L.hnext[threadIdx.x] = hs[threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
        L.scal[S_NRM2] = nrm;
        cgs_next_body(L, K - 1, p);
    }
}
template <typename C, int K>
__global__ void __launch_bounds__(kVT) k_cgs_pass_fused_t(const C *__restrict__ V, size_t ld, C *__restrict__ w,
                                                          size_t N, double2 *part, Level L, int p, const int *gate)
{
    if ((gate && *gate == 0) || L.flags[F_PASS] == 0) return;
    cgs_pass_body<C, K>(V, ld, w, N, part, L, p);
}
template <typename C, int K>
__global__ void __launch_bounds__(kVT) k_cgs_pass_fused_m(Multi<C> mm, size_t ld, size_t N, int p)
{
    const int y = blockIdx.y;
    if ((mm.gate[y] && *mm.gate[y] == 0) || mm.L[y].flags[F_PASS] == 0) return;
    Level L = mm.L[y];
    cgs_pass_body<C, K>(mm.V[y], ld, mm.w[y], N, mm.part[y], L, p);
}

// ||w||^2 into *nrm2
template <typename C>
__global__ void __launch_bounds__(kVT) k_norm2_fused(const C *__restrict__ w, size_t N, double2 *part, double *nrm2,
                                                     unsigned *counter, const int *gate)
{
    if (gate && *gate == 0) return;
    using R = typename RealOf<C>::T;
    using W = typename Wide<C>::T;
    constexpr int E = Wide<C>::E, U = 4;  // 16-byte words, U of them loaded before the first product
    R ax[1] = {R(0)}, ay[1] = {R(0)};
    const size_t S = (size_t)gridDim.x * kVT, t0 = blockIdx.x * (size_t)kVT + threadIdx.x;
    const size_t Nw = wide_words<C>(N, N);
    const W *__restrict__ ww = reinterpret_cast<const W *>(w);
    size_t i = t0;
    for (; i + (U - 1) * S < Nw; i += U * S) {
        W v[U];
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = ww[i + u * S];
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
            for (int e = 0; e < E; e++) {
                const C a = part_of(v[u], e);
                ax[0] += a.x * a.x + a.y * a.y;
            }
    }
    for (; i < Nw; i += S) {
        const W v = ww[i];
#pragma unroll
        for (int e = 0; e < E; e++) {
            const C a = part_of(v, e);
            ax[0] += a.x * a.x + a.y * a.y;
        }
    }
    for (i = Nw * E + t0; i < N; i += S) {
        const C wv = w[i];
        ax[0] += wv.x * wv.x + wv.y * wv.y;
    }
    block_reduce_store_r<0, R>(ax, ay, part);
    if (!last_block(counter)) return;
    __shared__ double nrm;
    reduce_partials(part, gridDim.x, 0, nullptr, &nrm);
    if (threadIdx.x == 0) *nrm2 = nrm;
}

// end of Arnoldi step j: V_{j+1} = w / ||w||, then the last block runs the Givens/misfit step
G2_D float2 scaled(float2 a, double s) { return make_float2((float)(a.x * s), (float)(a.y * s)); }
G2_D double2 scaled(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
G2_D double2 widen(float2 a) { return make_double2(a.x, a.y); }
G2_D double2 widen(double2 a) { return a; }

template <typename C>
G2_D void scale_finish_body(C *v, const C *w, size_t N, Level &L, int j, double tol)
{
    using W = typename Wide<C>::T;
    constexpr int E = Wide<C>::E;
    const double inv = 1.0 / L.scal[S_DNORMW];
    // kILP independent words per thread and iteration, loads first: more bytes in flight per SM
    const size_t S = (size_t)gridDim.x * kVT, t0 = blockIdx.x * (size_t)kVT + threadIdx.x;
    const size_t Nw = wide_words<C>(N, N);
    const W *__restrict__ ww = reinterpret_cast<const W *>(w);
    W *__restrict__ vw = reinterpret_cast<W *>(v);
    size_t i = t0;
    for (; i + (kILP - 1) * S < Nw; i += kILP * S) {
        W x[kILP];
#pragma unroll
        for (int u = 0; u < kILP; u++) x[u] = ww[i + u * S];
#pragma unroll
        for (int u = 0; u < kILP; u++) {
#pragma unroll
            for (int e = 0; e < E; e++) set_part(x[u], e, scaled(part_of(x[u], e), inv));
            vw[i + u * S] = x[u];
        }
    }
    for (; i < Nw; i += S) {
        W x = ww[i];
#pragma unroll
        for (int e = 0; e < E; e++) set_part(x, e, scaled(part_of(x, e), inv));
        vw[i] = x;
    }
    for (i = Nw * E + t0; i < N; i += S) v[i] = scaled(w[i], inv);
    if (!last_block(L.counter)) return;
    arnoldi_finish_body(L, j, tol);
}
template <typename C>
__global__ void __launch_bounds__(kVT) k_scale_finish(C *v, const C *w, size_t N, Level L, int j, double tol,
                                                      const int *gate)
{
    if (gate && *gate == 0) return;
    scale_finish_body<C>(v, w, N, L, j, tol);
}
// Multi: V[y] is the instance's basis, column j+1 is written
template <typename C>
__global__ void __launch_bounds__(kVT) k_scale_finish_m(Multi<C> mm, size_t N, int j, double tol)
{
    const int y = blockIdx.y;
    if (mm.gate[y] && *mm.gate[y] == 0) return;
    Level L = mm.L[y];
    scale_finish_body<C>(mm.V[y] + (size_t)(j + 1) * N, mm.w[y], N, L, j, tol);
}

// ConstructCurrentSolution's triangular solve (gmres.F90:441-445): y = H(0:L,0:L)^-1 g.  The block stages the
// L x L triangle and g in shared memory with one coalesced load; thread 0 then substitutes in the same order
// as the single-thread loop it replaces, so y is bit-for-bit the same (a chain of dependent L2 loads had made
// this 13 us per call).  Launch with kTriThreads threads.
constexpr int kTriThreads = 128;
__global__ void __launch_bounds__(kTriThreads) k_trisolve(Level L, const int *gate)
{
    if (gate && *gate == 0) return;
    __shared__ double2 Hs[KMAX * (KMAX + 1)];  // column j < n of the triangle at j * KMAX, then g at n * KMAX
    __shared__ double2 ys[KMAX];
    const int m = L.m, n = L.flags[F_L];
    for (int e = threadIdx.x; e < n * (n + 1); e += blockDim.x) {
        const int i = e % n, j = e / n, col = j < n ? j : m;
        Hs[i + j * KMAX] = L.H[hix(i, col, m)];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double2 *g = Hs + n * KMAX;
        for (int i = n - 1; i >= 0; i--) {
            double2 t = g[i];
            for (int k = i + 1; k < n; k++) {
                const double2 p = cmul_(Hs[i + k * KMAX], ys[k]);
                t.x -= p.x;
                t.y -= p.y;
            }
            const double2 d = Hs[i + i * KMAX];
            const double den = d.x * d.x + d.y * d.y;
            ys[i] = make_double2((t.x * d.x + t.y * d.y) / den, (t.y * d.x - t.x * d.y) / den);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) L.y[i] = ys[i];
}

// start of a cycle: H(0,m) = beta, H(1..m, m) = 0, krylov active (gmres.F90:172-185)
__global__ void k_cycle_start(Level L, const int *gate)
{
    if (gate && *gate == 0) return;
    const int m = L.m;
    L.H[hix(0, m, m)] = make_double2(L.scal[S_BETA], 0.0);
    for (int i = 1; i <= m; i++) L.H[hix(i, m, m)] = make_double2(0.0, 0.0);
    L.flags[F_KRYLOV] = 1;
    L.flags[F_L] = 0;
}

// inner solve start: bn from nrm2; beta from the residual; exit when beta/bn < tol (gmres.F90:139-168)
__global__ void k_set_bn(Level L)
{
    L.scal[S_BN] = sqrt(L.scal[S_NRM2]);
    L.flags[F_SOLVER] = L.scal[S_BN] < ZERO_THRESHOLD ? 0 : 1;
    L.flags[F_ITER] = 0;
    L.flags[F_KRYLOV] = L.flags[F_SOLVER];
    L.flags[F_L] = 0;
    L.flags[F_PASS] = 0;
}
__global__ void k_set_beta(Level L, double tol)
{
    if (L.flags[F_SOLVER] == 0) return;
    const double beta = sqrt(L.scal[S_NRM2]);
    L.scal[S_BETA] = beta;
    if (beta / L.scal[S_BN] < tol) {
        L.flags[F_SOLVER] = 0;
        L.flags[F_KRYLOV] = 0;
    }
}
__global__ void k_zero_level(Level L)
{
    const int n = (L.m + 1) * (L.m + 1);
    for (int i = threadIdx.x; i < n; i += blockDim.x) L.H[i] = make_double2(0.0, 0.0);
}

// restart (gmres.F90:369-376): beta = |g_m|, g <- inverse rotations of (0..0, g_m)
__global__ void k_restart_g(Level L)
{
    const int m = L.m;
    L.scal[S_BETA] = cabs_(L.H[hix(m, m, m)]);
    for (int J = m - 1; J >= 0; J--) {
        L.H[hix(J, m, m)] = make_double2(0.0, 0.0);
        zrot1(L.H[hix(J, m, m)], L.H[hix(J + 1, m, m)], L.cs[J], make_double2(-L.sn[J].x, -L.sn[J].y));
    }
    L.flags[F_L] = m + 1;  // the restart residual combines m+1 basis vectors with column m
}

// ---- vector kernels ----------------------------------------------------------------------------
// out = a*x + b*y (real scalars), x, y, out may differ in type
template <typename CO, typename CX, typename CY>
__global__ void __launch_bounds__(kVT) k_axpby(CO *out, double a, const CX *x, double b, const CY *y, size_t N,
                                               const int *gate)
{
    if (gate && *gate == 0) return;
    auto elem = [&](double2 xv, double2 yv) {
        double2 r = make_double2(a * xv.x, a * xv.y);
        if (y) {
            r.x += b * yv.x;
            r.y += b * yv.y;
        }
        return r;
    };
    // kILP independent elements per thread and iteration, loads first (out may alias x or y: every
    // element is still read before it is written, by the same thread)
    const size_t S = (size_t)gridDim.x * kVT;
    size_t i = blockIdx.x * (size_t)kVT + threadIdx.x;
    for (; i + (kILP - 1) * S < N; i += kILP * S) {
        double2 xv[kILP], yv[kILP];
#pragma unroll
        for (int u = 0; u < kILP; u++) {
            xv[u] = ld2(x, i + u * S);
            yv[u] = y ? ld2(y, i + u * S) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < kILP; u++) st2(out, i + u * S, elem(xv[u], yv[u]));
    }
    for (; i < N; i += S) st2(out, i, elem(ld2(x, i), y ? ld2(y, i) : make_double2(0.0, 0.0)));
}
// x = v, or x = 0 when ||v|| < ZERO_THRESHOLD (gmres.F90:139-145)
template <typename C>
__global__ void __launch_bounds__(kVT) k_copy_or_zero(C *x, const C *v, const double *scal, size_t N)
{
    const bool zero = scal[S_BN] < ZERO_THRESHOLD;
    for (size_t i = blockIdx.x * (size_t)kVT + threadIdx.x; i < N; i += (size_t)gridDim.x * kVT)
        st2(x, i, zero ? make_double2(0.0, 0.0) : ld2(v, i));
}
// v = w / scal[idx]
template <typename C>
__global__ void __launch_bounds__(kVT) k_scale_by(C *v, const C *w, const double *scal, int idx, size_t N,
                                                  const int *gate)
{
    if (gate && *gate == 0) return;
    const double inv = 1.0 / scal[idx];
    for (size_t i = blockIdx.x * (size_t)kVT + threadIdx.x; i < N; i += (size_t)gridDim.x * kVT) {
        const double2 x = ld2(w, i);
        st2(v, i, make_double2(x.x * inv, x.y * inv));
    }
}
// out = a0*in0 + sum_{k < n} B_k coef_k, n = flags[F_L] (or Kfix >= 0)
template <typename CO, typename CB>
__global__ void __launch_bounds__(kVT) k_lincomb(CO *out, double a0, const CO *in0, const CB *__restrict__ Bm,
                                                 size_t ld, const double2 *__restrict__ coef, const int *nflag,
                                                 size_t N, const int *gate)
{
    if (gate && *gate == 0) return;
    __shared__ double2 cs[KMAX + 1];
    const int n = *nflag;
    if (threadIdx.x < n) cs[threadIdx.x] = coef[threadIdx.x];
    __syncthreads();
    using W = typename Wide<CB>::T;
    constexpr int E = Wide<CB>::E;
    constexpr int KU = 4;  // basis words loaded together
    const size_t S = (size_t)gridDim.x * kVT, t0 = blockIdx.x * (size_t)kVT + threadIdx.x;
    const size_t Nw = wide_words<CB>(N, ld), ldw = ld / E;
    const W *__restrict__ Bw = reinterpret_cast<const W *>(Bm);
    size_t i = t0;
    for (; i < Nw; i += S) {
        double2 r[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
            r[e] = make_double2(0.0, 0.0);
            if (in0) {
                const double2 x = ld2(in0, i * E + e);
                r[e] = make_double2(a0 * x.x, a0 * x.y);
            }
        }
        int k = 0;
        for (; k + KU <= n; k += KU) {
            W v[KU];
#pragma unroll
            for (int q = 0; q < KU; q++) v[q] = Bw[(size_t)(k + q) * ldw + i];
#pragma unroll
            for (int q = 0; q < KU; q++)
#pragma unroll
                for (int e = 0; e < E; e++) {
                    const double2 b = widen(part_of(v[q], e)), c = cs[k + q];
                    r[e].x += b.x * c.x - b.y * c.y;
                    r[e].y += b.x * c.y + b.y * c.x;
                }
        }
        for (; k < n; k++) {
            const W v = Bw[(size_t)k * ldw + i];
#pragma unroll
            for (int e = 0; e < E; e++) {
                const double2 b = widen(part_of(v, e)), c = cs[k];
                r[e].x += b.x * c.x - b.y * c.y;
                r[e].y += b.x * c.y + b.y * c.x;
            }
        }
#pragma unroll
        for (int e = 0; e < E; e++) st2(out, i * E + e, r[e]);
    }
    for (i = Nw * E + t0; i < N; i += S) {
        double2 r = make_double2(0.0, 0.0);
        if (in0) {
            const double2 x = ld2(in0, i);
            r = make_double2(a0 * x.x, a0 * x.y);
        }
        for (int k = 0; k < n; k++) {
            const double2 v = ld2(Bm, (size_t)k * ld + i);
            r.x += v.x * cs[k].x - v.y * cs[k].y;
            r.y += v.x * cs[k].y + v.y * cs[k].x;
        }
        st2(out, i, r);
    }
}
// copy the g column into a coefficient vector (restart residual w = V g)
__global__ void k_copy_g(Level L)
{
    const int m = L.m;
    for (int i = threadIdx.x; i <= m; i += blockDim.x) L.y[i] = L.H[hix(i, m, m)];
}

// SolveEquation helpers (ie_solver_module.F90:64-97); vectors are [c][cell], cell = z*NxNy + y*Nx + x
__global__ void k_rhs(double2 *rhs, const double2 *Ebkg, const double *post, size_t plane, int Nz)
{
    const size_t n = 3 * plane * Nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)((i / plane) % Nz);
        rhs[i] = make_double2(post[z] * Ebkg[i].x, post[z] * Ebkg[i].y);
    }
}
__global__ void k_scale_asig(double2 *out, const double2 *in, const double2 *asig, size_t cells, bool divide)
{
    const size_t n = 3 * cells;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double2 a = asig[i % cells];
        const double2 v = in[i];
        if (divide) {
            const double den = a.x * a.x + a.y * a.y;
            out[i] = make_double2((v.x * a.x + v.y * a.y) / den, (v.y * a.x - v.x * a.y) / den);
        } else {
            out[i] = make_double2(v.x * a.x - v.y * a.y, v.x * a.y + v.y * a.x);
        }
    }
}

int vec_grid(size_t N)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const size_t need = (N + kVT - 1) / kVT;
    const size_t g = (size_t)sms * 4;
    return (int)(need < g ? need : g);
}
// blocks of the sweeps that end in a last-block reduction: two per SM and instance streamed as fast as
// four in the basis sweeps, and leave the last block half as many partial sums to add
int sweep_grid(size_t N)
{
    const int g = vec_grid(N);
    return g > 8 ? (g + 1) / 2 : g;
}

}  // namespace

// --------------------------------------------------------------------------------------------------
struct KrylovWork {
    size_t N = 0;
    int mo = 0, mi = 0, precision = -1;
    // outer (FP64)
    double2 *Vo = nullptr, *x = nullptr, *b = nullptr, *r0 = nullptr, *w = nullptr, *tmp = nullptr;
    void *Zo = nullptr;  // complex128 (plain) or complex64 (mixed)
    // inner
    void *Vi = nullptr, *ri = nullptr, *wi = nullptr, *vin = nullptr, *xin = nullptr;
    Level Lo, Li;
    // the inner GMRES cycle as CUDA graphs (fixed buffers vin -> xin; slot 0 starts at x0 = vin as the
    // reference does, slot 1 at x0 = x0in, the outer preconditioner hook's guess), captured on second use
    cudaGraphExec_t inner_exec[2] = {nullptr, nullptr};
    double inner_tol[2] = {-1.0, -1.0};
    int inner_uses[2] = {0, 0}, inner_graph_applies[2] = {0, 0}, inner_graph_launches[2] = {0, 0};
    bool inner_true_res[2] = {false, false};
    long long inner_gen[2] = {-1, -1};          // operator launch configuration baked into the graphs
    void *x0in = nullptr;                       // warm start of the inner cycle (inner precision)
    double2 *part = nullptr;
    int nparts = 0;
    std::vector<double> history;
    int applies64 = 0, applies32 = 0;
    int hook_steps = 0;  // outer steps preconditioned through the hook in the last solve
};

static int alloc_level(Level &L, int m)
{
    L.m = m;
    G2_CUDA_CHECK(cudaMalloc(&L.H, sizeof(double2) * (m + 1) * (m + 1)));
    G2_CUDA_CHECK(cudaMalloc(&L.cs, sizeof(double) * (m + 1)));
    G2_CUDA_CHECK(cudaMalloc(&L.sn, sizeof(double2) * (m + 1)));
    G2_CUDA_CHECK(cudaMalloc(&L.hpass, sizeof(double2) * (KMAX + 1)));
    G2_CUDA_CHECK(cudaMalloc(&L.hnext, sizeof(double2) * (KMAX + 1)));
    G2_CUDA_CHECK(cudaMalloc(&L.y, sizeof(double2) * (KMAX + 1)));
    G2_CUDA_CHECK(cudaMalloc(&L.scal, sizeof(double) * S_NSCAL));
    G2_CUDA_CHECK(cudaMalloc(&L.flags, sizeof(int) * F_NFLAGS));
    G2_CUDA_CHECK(cudaMalloc(&L.counter, sizeof(unsigned)));
    G2_CUDA_CHECK(cudaMemset(L.counter, 0, sizeof(unsigned)));
    G2_CUDA_CHECK(cudaMemset(L.flags, 0, sizeof(int) * F_NFLAGS));
    G2_CUDA_CHECK(cudaMemset(L.scal, 0, sizeof(double) * S_NSCAL));
    // the solver's kernels run on non-blocking streams, which are not ordered after the legacy stream
    G2_CUDA_CHECK(cudaStreamSynchronize(cudaStreamLegacy));
    return G2_OK;
}
static void free_level(Level &L)
{
    void *p[] = {L.H, L.cs, L.sn, L.hpass, L.hnext, L.y, L.scal, L.flags, L.counter};
    for (void *q : p)
        if (q) cudaFree(q);
    L = Level();
}

static void kw_free(KrylovWork *k)
{
    if (!k) return;
    for (int q = 0; q < 2; q++)
        if (k->inner_exec[q]) cudaGraphExecDestroy(k->inner_exec[q]);
    void *p[] = {k->Vo, k->x, k->b, k->r0, k->w, k->tmp, k->Zo, k->Vi, k->ri, k->wi, k->vin, k->xin, k->part, k->x0in};
    for (void *q : p)
        if (q) cudaFree(q);
    free_level(k->Lo);
    free_level(k->Li);
    delete k;
}

void krylov_free(IeOp *op)
{
    kw_free(reinterpret_cast<KrylovWork *>(op->krylov));
    op->krylov = nullptr;
}

// solver workspace for vectors of N complex: outer basis mo, inner basis mi
static int kw_alloc(KrylovWork *k, size_t N, int mo, int mi, int precision)
{
    k->N = N;
    k->mo = mo;
    k->mi = mi;
    k->precision = precision;
    const size_t e64 = sizeof(double2), ei = precision ? sizeof(float2) : sizeof(double2);
    G2_CUDA_CHECK(cudaMalloc(&k->Vo, e64 * N * (mo + 1)));
    G2_CUDA_CHECK(cudaMalloc(&k->x, e64 * N));
    G2_CUDA_CHECK(cudaMalloc(&k->b, e64 * N));
    G2_CUDA_CHECK(cudaMalloc(&k->r0, e64 * N));
    G2_CUDA_CHECK(cudaMalloc(&k->w, e64 * N));
    G2_CUDA_CHECK(cudaMalloc(&k->tmp, e64 * N));
    G2_CUDA_CHECK(cudaMalloc(&k->Zo, ei * N * mo));
    G2_CUDA_CHECK(cudaMalloc(&k->Vi, ei * N * (mi + 1)));
    G2_CUDA_CHECK(cudaMalloc(&k->ri, ei * N));
    G2_CUDA_CHECK(cudaMalloc(&k->wi, ei * N));
    G2_CUDA_CHECK(cudaMalloc(&k->vin, ei * N));
    G2_CUDA_CHECK(cudaMalloc(&k->xin, ei * N));
    G2_CUDA_CHECK(cudaMalloc(&k->x0in, ei * N));
    k->nparts = sweep_grid(N);
    G2_CUDA_CHECK(cudaMalloc(&k->part, sizeof(double2) * (size_t)k->nparts * (KMAX + 1)));
    int rc = alloc_level(k->Lo, mo);
    if (!rc) rc = alloc_level(k->Li, mi);
    return rc;
}

static int krylov_alloc(IeOp *op, int mo, int mi, int precision)
{
    KrylovWork *k = reinterpret_cast<KrylovWork *>(op->krylov);
    if (k && k->mo == mo && k->mi == mi && k->precision == precision) return G2_OK;
    krylov_free(op);
    k = new KrylovWork();
    op->krylov = k;
    return kw_alloc(k, op->nvec(), mo, mi, precision);
}

// ---- launch helpers ------------------------------------------------------------------------------
// Blocks per instance of a sweep: whole waves of the instantiation's resident blocks, as near as possible to
// `want` (the instance's partial-sum slots, never more).  A grid that asks for 4 blocks per SM of a kernel
// that fits 3 runs a last wave at a third of the bytes in flight: the FP64 first-dots sweep (80 registers)
// streamed at 2.6 TB/s that way against 5 TB/s for the same data in the correction pass.
static int sm_count()
{
    static const int sms = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n > 0 ? n : 1;
    }();
    return sms;
}
template <class F> static int resident_blocks(F fn)
{
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kVT, 0) != cudaSuccess || b < 1) b = 1;
    return b;
}
static int wave_grid(int per_sm, int want, int ninst)
{
    const int wave = per_sm * sm_count(), total = want * ninst;
    int waves = (total + wave / 2) / wave;
    if (waves < 1) waves = 1;
    const int g = waves * wave / ninst;
    return g < 1 ? 1 : (g < want ? g : want);
}
template <typename C, int K>
static void launch_dots_first_k(KrylovWork *k, const C *V, const C *w, Level &L, const int *g, cudaStream_t st)
{
    static const int per_sm = resident_blocks(k_dots_first_t<C, K>);
    k_dots_first_t<C, K><<<wave_grid(per_sm, k->nparts, 1), kVT, 0, st>>>(V, k->N, w, k->N, k->part, L, g);
}
template <typename C, int K>
static void launch_pass_fused_k(KrylovWork *k, const C *V, C *w, Level &L, int p, const int *g, cudaStream_t st)
{
    k_cgs_pass_fused_t<C, K><<<k->nparts, kVT, 0, st>>>(V, k->N, w, k->N, k->part, L, p, g);
}
#define G2_KCASES(F, ...)                                                                                     \
    switch (K) {                                                                                          \
    case 0: F<C, 0>(__VA_ARGS__); break; case 1: F<C, 1>(__VA_ARGS__); break;                             \
    case 2: F<C, 2>(__VA_ARGS__); break; case 3: F<C, 3>(__VA_ARGS__); break;                             \
    case 4: F<C, 4>(__VA_ARGS__); break; case 5: F<C, 5>(__VA_ARGS__); break;                             \
    case 6: F<C, 6>(__VA_ARGS__); break; case 7: F<C, 7>(__VA_ARGS__); break;                             \
    case 8: F<C, 8>(__VA_ARGS__); break; case 9: F<C, 9>(__VA_ARGS__); break;                             \
    case 10: F<C, 10>(__VA_ARGS__); break; case 11: F<C, 11>(__VA_ARGS__); break;                         \
    case 12: F<C, 12>(__VA_ARGS__); break; case 13: F<C, 13>(__VA_ARGS__); break;                         \
    case 14: F<C, 14>(__VA_ARGS__); break; case 15: F<C, 15>(__VA_ARGS__); break;                         \
    case 16: F<C, 16>(__VA_ARGS__); break; case 17: F<C, 17>(__VA_ARGS__); break;                         \
    case 18: F<C, 18>(__VA_ARGS__); break; case 19: F<C, 19>(__VA_ARGS__); break;                         \
    case 20: F<C, 20>(__VA_ARGS__); break; case 21: F<C, 21>(__VA_ARGS__); break;                         \
    case 22: F<C, 22>(__VA_ARGS__); break; case 23: F<C, 23>(__VA_ARGS__); break;                         \
    case 24: F<C, 24>(__VA_ARGS__); break; case 25: F<C, 25>(__VA_ARGS__); break;                         \
    case 26: F<C, 26>(__VA_ARGS__); break; case 27: F<C, 27>(__VA_ARGS__); break;                         \
    case 28: F<C, 28>(__VA_ARGS__); break; case 29: F<C, 29>(__VA_ARGS__); break;                         \
    case 30: F<C, 30>(__VA_ARGS__); break; case 31: F<C, 31>(__VA_ARGS__); break;                         \
    default: F<C, 32>(__VA_ARGS__); break;                                                                \
    }

template <typename C>
static void norm2(KrylovWork *k, const C *w, double *nrm2, const int *g, cudaStream_t st)
{
    // kernels on one stream run one after another, so any level's counter serves
    k_norm2_fused<C><<<k->nparts, kVT, 0, st>>>(w, k->N, k->part, nrm2, k->Lo.counter, g); g2_count_launches(1);
}

// CGS for Arnoldi step j on level L with basis V (j+1 columns) and vector w: the first pass's dots and
// up to N_IGS+1 correction passes, each one launch (passes after the decision to stop exit at once)
template <typename C>
static void cgs(KrylovWork *k, Level &L, const C *V, int j, C *w, const int *gate, cudaStream_t st)
{
    const int K = j + 1;
    G2_KCASES(launch_dots_first_k, k, V, w, L, gate, st)
    g2_count_launches(1);
    for (int p = 1; p <= N_IGS + 1; p++) {
        G2_KCASES(launch_pass_fused_k, k, V, w, L, p, gate, st)
        g2_count_launches(1);
    }
}
// end of Arnoldi step j: V_{j+1} = w / ||w|| and the Givens / misfit update, one launch
template <typename C>
static void arnoldi_tail(KrylovWork *k, Level &L, C *V, int j, const C *w, double tol, const int *gate, cudaStream_t st)
{
    k_scale_finish<C><<<sweep_grid(k->N), kVT, 0, st>>>(V + (size_t)(j + 1) * k->N, w, k->N, L, j, tol, gate);
    g2_count_launches(1);
}

// the same CGS and Arnoldi tail for n lockstep instances (vector length N, nparts blocks each) in one
// launch per kernel
template <typename C, int K>
static void launch_dots_first_km(const Multi<C> &mm, int n, size_t N, int nparts, cudaStream_t st)
{
    static const int per_sm = resident_blocks(k_dots_first_m<C, K>);
    k_dots_first_m<C, K><<<dim3(wave_grid(per_sm, nparts, n), n), kVT, 0, st>>>(mm, N, N);
}
template <typename C, int K>
static void launch_pass_fused_km(const Multi<C> &mm, int n, size_t N, int nparts, int p, cudaStream_t st)
{
    k_cgs_pass_fused_m<C, K><<<dim3(nparts, n), kVT, 0, st>>>(mm, N, N, p);
}
template <typename C>
static void cgs_multi(const Multi<C> &mm, int n, size_t N, int nparts, int j, cudaStream_t st)
{
    const int K = j + 1;
    G2_KCASES(launch_dots_first_km, mm, n, N, nparts, st)
    g2_count_launches(1);
    for (int p = 1; p <= N_IGS + 1; p++) {
        G2_KCASES(launch_pass_fused_km, mm, n, N, nparts, p, st)
        g2_count_launches(1);
    }
}
template <typename C>
static void arnoldi_tail_multi(const Multi<C> &mm, int n, size_t N, int j, double tol, cudaStream_t st)
{
    k_scale_finish_m<C><<<dim3(sweep_grid(N), n), kVT, 0, st>>>(mm, N, j, tol);
    g2_count_launches(1);
}

template <typename C> static int apply_prec(IeOp *op, const C *in, C *out, cudaStream_t st, const int *gate);
template <> int apply_prec<double2>(IeOp *op, const double2 *in, double2 *out, cudaStream_t st, const int *gate)
{
    return ie_apply_device64(op, in, out, st, gate);
}
template <> int apply_prec<float2>(IeOp *op, const float2 *in, float2 *out, cudaStream_t st, const int *gate)
{
    return ie_apply_device32(op, in, out, st, gate);
}

// Inner GMRES (seq_fgmres.F90:142-152 -> gmres.F90:110-213 with MaxIt = 1, x0 = b = v): x = M(v)
template <typename CI>
static int inner_solve(IeOp *op, KrylovWork *k, const CI *v, const CI *x0, CI *x, double tol, bool true_residual,
                       cudaStream_t st)
{
    Level &L = k->Li;
    const size_t N = k->N;
    const int g = vec_grid(N);
    CI *Vi = reinterpret_cast<CI *>(k->Vi), *ri = reinterpret_cast<CI *>(k->ri), *wi = reinterpret_cast<CI *>(k->wi);
    const int *solver = L.flags + F_SOLVER, *krylov = L.flags + F_KRYLOV;
    k_zero_level<<<1, 256, 0, st>>>(L); g2_count_launches(1);
    norm2<CI>(k, v, L.scal + S_NRM2, nullptr, st);
    k_set_bn<<<1, 1, 0, st>>>(L); g2_count_launches(1);
    k_copy_or_zero<CI><<<g, kVT, 0, st>>>(x, x0, L.scal, N);  // x = x0, or 0 when ||b|| < 1e-14
    int rc = apply_prec<CI>(op, x0, ri, st, solver);
    if (rc) return rc;
    k->applies32 += sizeof(CI) == 8 ? 1 : 0;
    k->applies64 += sizeof(CI) == 16 ? 1 : 0;
    k_axpby<CI, CI, CI><<<g, kVT, 0, st>>>(ri, 1.0, v, -1.0, ri, N, solver);  // r0 = b - A x0
    norm2<CI>(k, ri, L.scal + S_NRM2, solver, st);
    k_set_beta<<<1, 1, 0, st>>>(L, tol); g2_count_launches(1);
    k_cycle_start<<<1, 1, 0, st>>>(L, solver); g2_count_launches(1);
    k_scale_by<CI><<<g, kVT, 0, st>>>(Vi, ri, L.scal, S_BETA, N, solver); g2_count_launches(1);
    for (int j = 0; j < k->mi; j++) {
        CI *Vj = Vi + (size_t)j * N;
        rc = apply_prec<CI>(op, Vj, wi, st, krylov);
        if (rc) return rc;
        k->applies32 += sizeof(CI) == 8 ? 1 : 0;
        k->applies64 += sizeof(CI) == 16 ? 1 : 0;
        cgs<CI>(k, L, Vi, j, wi, krylov, st);
        arnoldi_tail<CI>(k, L, Vi, j, wi, tol, krylov, st);
    }
    // FinalActions -> ConstructCurrentSolution (gmres.F90:423-458): x = x0 + V y
    k_trisolve<<<1, kTriThreads, 0, st>>>(L, solver); g2_count_launches(1);
    k_lincomb<CI, CI><<<g, kVT, 0, st>>>(x, 1.0, x, Vi, N, L.y, L.flags + F_L, N, solver); g2_count_launches(1);
    if (true_residual) {  // gmres.F90:402-419, result unused by the outer solver
        rc = apply_prec<CI>(op, x, ri, st, solver);
        if (rc) return rc;
        k->applies32 += sizeof(CI) == 8 ? 1 : 0;
        k->applies64 += sizeof(CI) == 16 ? 1 : 0;
    }
    return G2_OK;
}

// inner solve vin -> xin (warm: starting at x0in); eager on first use, then captured once and replayed
template <typename CI>
static int inner_solve_fixed(IeOp *op, KrylovWork *k, double tol, bool true_res, bool warm, cudaStream_t st)
{
    const int q = warm ? 1 : 0;
    const CI *v = reinterpret_cast<const CI *>(k->vin);
    const CI *x0 = warm ? reinterpret_cast<const CI *>(k->x0in) : v;
    CI *x = reinterpret_cast<CI *>(k->xin);
    const char *ng = std::getenv("GIEM2G_NO_GRAPHS");
    const bool graphs = !(ng && ng[0] == '1');
    if (k->inner_exec[q] && (k->inner_tol[q] != tol || k->inner_true_res[q] != true_res ||
                             k->inner_gen[q] != op->config_gen)) {
        cudaGraphExecDestroy(k->inner_exec[q]);
        k->inner_exec[q] = nullptr;
        k->inner_uses[q] = 0;
    }
    auto credit = [&]() {
        g2_count_launches(k->inner_graph_launches[q]);
        if (sizeof(CI) == 8) k->applies32 += k->inner_graph_applies[q];
        else k->applies64 += k->inner_graph_applies[q];
    };
    if (k->inner_exec[q]) {
        G2_CUDA_CHECK(cudaGraphLaunch(k->inner_exec[q], st));
        credit();
        return G2_OK;
    }
    if (!graphs || k->inner_uses[q]++ == 0) return inner_solve<CI>(op, k, v, x0, x, tol, true_res, st);
    // capture: count what one cycle launches, then instantiate
    const int a32 = k->applies32, a64 = k->applies64;
    const long long l0 = g2_launch_total();
    cudaGraph_t graph = nullptr;
    G2_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = inner_solve<CI>(op, k, v, x0, x, tol, true_res, st);
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (rc) return rc;
    if (ce != cudaSuccess) {
        g2_set_error(__FILE__, __LINE__, cudaGetErrorString(ce));
        return G2_ERR_CUDA;
    }
    k->inner_graph_applies[q] = (k->applies32 - a32) + (k->applies64 - a64);
    k->inner_graph_launches[q] = (int)(g2_launch_total() - l0);
    k->applies32 = a32;
    k->applies64 = a64;
    ce = cudaGraphInstantiate(&k->inner_exec[q], graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
        g2_set_error(__FILE__, __LINE__, cudaGetErrorString(ce));
        k->inner_exec[q] = nullptr;
        return G2_ERR_CUDA;
    }
    k->inner_tol[q] = tol;
    k->inner_true_res[q] = true_res;
    k->inner_gen[q] = op->config_gen;
    G2_CUDA_CHECK(cudaGraphLaunch(k->inner_exec[q], st));
    credit();
    return G2_OK;
}

template <typename CI>
static int outer_solve(IeOp *op, KrylovWork *k, const GIEM2G_FGMRES_CTL &ctl, GIEM2G_RESULT *info, cudaStream_t st)
{
    Level &L = k->Lo;
    const size_t N = k->N;
    const int g = vec_grid(N), M = k->mo;
    const double tol = ctl.misfit;
    const char *tr = std::getenv("GIEM2G_INNER_TRUE_RESIDUAL");
    const bool true_res = tr && tr[0] == '1';
    CI *Z = reinterpret_cast<CI *>(k->Zo);
    CI *vin = reinterpret_cast<CI *>(k->vin);
    double h_scal[S_NSCAL];
    int h_flags[F_NFLAGS];
    auto pull = [&]() -> int {
        G2_CUDA_CHECK(cudaMemcpyAsync(h_scal, L.scal, sizeof(h_scal), cudaMemcpyDeviceToHost, st));
        G2_CUDA_CHECK(cudaMemcpyAsync(h_flags, L.flags, sizeof(h_flags), cudaMemcpyDeviceToHost, st));
        G2_CUDA_CHECK(cudaStreamSynchronize(st));
        return ie_check_device_error(op);
    };
    k->history.clear();
    info->iterations = 0;
    info->bea = -1.0;
    info->be = -1.0;
    // gmres.F90:129-168
    k_zero_level<<<1, 256, 0, st>>>(L); g2_count_launches(1);
    norm2<double2>(k, k->b, L.scal + S_NRM2, nullptr, st);
    k_set_bn<<<1, 1, 0, st>>>(L); g2_count_launches(1);
    int rc = pull();
    if (rc) return rc;
    if (h_scal[S_BN] < ZERO_THRESHOLD) {
        cudaMemsetAsync(k->x, 0, sizeof(double2) * N, st);
        info->stat = 1;
        return G2_OK;
    }
    const double bn = h_scal[S_BN];
    rc = ie_apply_device64(op, k->x, k->r0, st);  // x holds x0
    if (rc) return rc;
    k->applies64++;
    k_axpby<double2, double2, double2><<<g, kVT, 0, st>>>(k->r0, 1.0, k->b, -1.0, k->r0, N, nullptr); g2_count_launches(1);
    k_axpby<double2, double2, double2><<<g, kVT, 0, st>>>(k->w, 1.0, k->r0, 0.0, (const double2 *)nullptr, N, nullptr); g2_count_launches(1);
    norm2<double2>(k, k->w, L.scal + S_NRM2, nullptr, st);
    k_set_beta<<<1, 1, 0, st>>>(L, tol); g2_count_launches(1);
    if ((rc = pull())) return rc;
    if (h_scal[S_BETA] / bn < tol) {
        info->stat = 1;
        info->be = h_scal[S_BETA] / bn;
        return G2_OK;
    }
    int iter = 0, L_used = 0;
    bool converged = false, hook_off = false;
    k->hook_steps = 0;
    double bea = -1.0;
    char msg[256];
    for (;;) {
        k_cycle_start<<<1, 1, 0, st>>>(L, nullptr); g2_count_launches(1);
        k_scale_by<double2><<<g, kVT, 0, st>>>(k->Vo, k->w, L.scal, S_BETA, N, nullptr); g2_count_launches(1);
        for (int j = 0; j < M; j++) {
            const double2 *Vj = k->Vo + (size_t)j * N;
            CI *Zj = Z + (size_t)j * N;
            // right preconditioner: Z_j = inner GMRES(V_j)  (gmres.F90:251, :491-506), through the fixed
            // buffers vin -> xin of the captured inner cycle.  With an outer preconditioner hook the hook's
            // output (complex128 in tmp) either starts the inner cycle (mode 1) or is Z_j itself (mode 2).
            bool hooked = false;
            if (op->precond_mode && !hook_off) {
                const int hr = op->precond_fn(op->precond_user, Vj, k->tmp, (long long)N, reinterpret_cast<void *>(st));
                if (hr == 0) hooked = true;
                else hook_off = true;
            }
            if (hooked && op->precond_mode == 2) {
                k_axpby<CI, double2, double2><<<g, kVT, 0, st>>>(Zj, 1.0, k->tmp, 0.0, (const double2 *)nullptr, N, nullptr); g2_count_launches(1);
            } else {
                k_axpby<CI, double2, double2><<<g, kVT, 0, st>>>(vin, 1.0, Vj, 0.0, (const double2 *)nullptr, N, nullptr); g2_count_launches(1);
                if (hooked) {
                    k_axpby<CI, double2, double2><<<g, kVT, 0, st>>>(reinterpret_cast<CI *>(k->x0in), 1.0, k->tmp, 0.0,
                                                                     (const double2 *)nullptr, N, nullptr); g2_count_launches(1);
                }
                if ((rc = inner_solve_fixed<CI>(op, k, tol, true_res, hooked, st))) return rc;
                k_axpby<CI, CI, CI><<<g, kVT, 0, st>>>(Zj, 1.0, reinterpret_cast<const CI *>(k->xin), 0.0, (const CI *)nullptr, N, nullptr); g2_count_launches(1);
            }
            if (sizeof(CI) == sizeof(double2)) {
                if ((rc = ie_apply_device64(op, reinterpret_cast<const double2 *>(Zj), k->w, st))) return rc;
            } else {
                k_axpby<double2, CI, CI><<<g, kVT, 0, st>>>(k->tmp, 1.0, Zj, 0.0, (const CI *)nullptr, N, nullptr); g2_count_launches(1);
                if ((rc = ie_apply_device64(op, k->tmp, k->w, st))) return rc;
            }
            k->applies64++;
            cgs<double2>(k, L, k->Vo, j, k->w, nullptr, st);
            arnoldi_tail<double2>(k, L, k->Vo, j, k->w, tol, nullptr, st);
            if ((rc = pull())) return rc;
            bea = h_scal[S_BEA];
            if (!std::isfinite(bea)) {
                g2_set_error_msg("FGMRES: non-finite Arnoldi misfit");
                return G2_ERR_NUMERIC;
            }
            // the hook must keep reducing the FP64 residual; otherwise the plain inner GMRES takes over
            if (hooked && !k->history.empty() && !(bea < kHookGain * k->history.back())) hook_off = true;
            if (hooked) k->hook_steps++;
            k->history.push_back(bea);
            info->iterations = (int)k->history.size();
            // ie_solver_module.F90:335-343 Information
            std::snprintf(msg, sizeof(msg), "FGMRES outer  iteration:%5d Arnoldy misfit: %10.3E", (int)k->history.size(), bea);
            g2_log(msg);
            L_used = j + 1;
            if (bea < tol) { converged = true; break; }
        }
        if (converged) break;
        iter++;
        if (iter >= ctl.fgmres_maxit) break;
        // PrepareRestart: x += Z y; w = V g' (gmres.F90:333-379)
        k_trisolve<<<1, kTriThreads, 0, st>>>(L, nullptr); g2_count_launches(1);
        k_lincomb<double2, CI><<<g, kVT, 0, st>>>(k->x, 1.0, k->x, Z, N, L.y, L.flags + F_L, N, nullptr); g2_count_launches(1);
        k_restart_g<<<1, 1, 0, st>>>(L); g2_count_launches(1);
        k_copy_g<<<1, 64, 0, st>>>(L); g2_count_launches(1);
        k_lincomb<double2, double2><<<g, kVT, 0, st>>>(k->w, 0.0, (const double2 *)nullptr, k->Vo, N, L.y,
                                                       L.flags + F_L, N, nullptr);
    }
    (void)L_used;
    // FinalActions (gmres.F90:382-421)
    k_trisolve<<<1, kTriThreads, 0, st>>>(L, nullptr); g2_count_launches(1);
    k_lincomb<double2, CI><<<g, kVT, 0, st>>>(k->x, 1.0, k->x, Z, N, L.y, L.flags + F_L, N, nullptr); g2_count_launches(1);
    if ((rc = ie_apply_device64(op, k->x, k->r0, st))) return rc;
    k->applies64++;
    k_axpby<double2, double2, double2><<<g, kVT, 0, st>>>(k->r0, 1.0, k->b, -1.0, k->r0, N, nullptr); g2_count_launches(1);
    norm2<double2>(k, k->r0, L.scal + S_NRM2, nullptr, st);
    if ((rc = pull())) return rc;
    const double be = std::sqrt(h_scal[S_NRM2]) / bn;
    info->iterations = (int)k->history.size();
    info->bea = bea;
    info->be = be;
    if (converged) info->stat = be >= tol ? 2 : 1;
    else info->stat = -1;
    return G2_OK;
}

int krylov_solve_device(IeOp *op, const double2 *d_Ebkg, double2 *d_Esol, const double2 *d_E0,
                        const GIEM2G_FGMRES_CTL &ctl, GIEM2G_RESULT *info)
{
    if (ctl.fgmres_buf < 1 || ctl.gmres_buf < 1 || ctl.fgmres_buf > KMAX - 1 || ctl.gmres_buf > KMAX - 1) {
        g2_set_error_msg("FGMRES buffer sizes must be in [1, 31]");
        return G2_ERR_UNSUPPORTED;
    }
    if (ctl.precision < 0 || ctl.precision > 1) return G2_ERR_ARG;
    int rc = krylov_alloc(op, ctl.fgmres_buf, ctl.gmres_buf, ctl.precision);
    if (rc) return rc;
    KrylovWork *k = reinterpret_cast<KrylovWork *>(op->krylov);
    cudaStream_t st = op->stream;
    const size_t cells = op->cells();
    const int g = vec_grid(k->N);
    k->applies32 = k->applies64 = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    // SolveEquation (ie_solver_module.F90:62-80): rhs = sqrt(Re sb) E_bkg; guess = E0/a or rhs
    k_rhs<<<g, 256, 0, st>>>(k->b, d_Ebkg, op->d_post64, (size_t)op->Nx * op->Ny, op->Nz); g2_count_launches(1);
    if (d_E0) {
        k_scale_asig<<<g, 256, 0, st>>>(k->x, d_E0, op->d_asig64, cells, true);
        g2_count_launches(1);
    } else {
        cudaMemcpyAsync(k->x, k->b, sizeof(double2) * k->N, cudaMemcpyDeviceToDevice, st);
    }
    if (ctl.precision == 0) rc = outer_solve<double2>(op, k, ctl, info, st);
    else rc = outer_solve<float2>(op, k, ctl, info, st);
    if (rc) return rc;
    // Esol = a * chi (ie_solver_module.F90:85-97)
    k_scale_asig<<<g, 256, 0, st>>>(d_Esol, k->x, op->d_asig64, cells, false); g2_count_launches(1);
    cudaEventRecord(e1, st);
    G2_CUDA_CHECK(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    info->applies_fp64 = k->applies64;
    info->applies_fp32 = k->applies32;
    info->precond_steps = k->hook_steps;
    info->device_ms = ms;
    op->mult_num += k->applies64 + k->applies32;
    op->apply_seconds += ms * 1e-3;
    return ie_check_device_error(op);
}

int krylov_history(IeOp *op, double *out, int max_len)
{
    KrylovWork *k = reinterpret_cast<KrylovWork *>(op->krylov);
    if (!k) return 0;
    const int n = (int)k->history.size() < max_len ? (int)k->history.size() : max_len;
    for (int i = 0; i < n; i++) out[i] = k->history[i];
    return n;
}

// ==================================================================================================
// Batched solves (several frequencies and both polarisations): n independent instances, each a full
// nested FGMRES with its own workspace, advanced in lockstep on one stream.  Per outer step the host
// launches every active instance's work, replays ONE captured inner cycle for all instances and reads
// all instances' scalars with one synchronisation.  Consecutive instances of the same operator form
// pairs whose complex64 applies share every tensor read (ie_apply_pair32).  Each instance follows exactly
// the launch sequence of the single solve, so its iterates, iteration count and status are those of a
// solve on its own.  Converged instances are masked: their inner-cycle kernels are gated off through a
// device flag and the host stops launching their outer work.
namespace {

// outer_go: the instance's outer Krylov flag (F_KRYLOV of its outer level); an inner cycle enqueued after the
// instance converged (one outer step ahead of the host, see batch_outer) does nothing.  (Masked instances
// launch nothing: each mask has its own captured cycle.)
__global__ void k_set_bn_masked(Level L, const int *outer_go)
{
    L.scal[S_BN] = sqrt(L.scal[S_NRM2]);
    L.flags[F_SOLVER] = (L.scal[S_BN] < ZERO_THRESHOLD || *outer_go == 0) ? 0 : 1;
    L.flags[F_ITER] = 0;
    L.flags[F_KRYLOV] = L.flags[F_SOLVER];
    L.flags[F_L] = 0;
    L.flags[F_PASS] = 0;
}

}  // namespace

struct BatchGroup {
    IeOp *op = nullptr;
    int first = 0, n = 0;  // instances first .. first+n-1 (n = 1 or 2)
};

struct BatchWork {
    int n = 0, mo = 0, mi = 0, precision = -1;
    std::vector<IeOp *> ops;
    std::vector<KrylovWork *> k;
    std::vector<BatchGroup> groups;
    std::vector<int> h_active;  // instances still running (each mask has its own captured inner cycle)
    double2 *d_stage = nullptr;  // host-array solves: E_bkg[n] then E_sol[n] (complex128)
    // pinned host copies of the outer levels' scalars and flags, two slots (outer step j uses slot j % 2),
    // each completed by its own event
    void *h_pin = nullptr;
    cudaEvent_t ev_pull[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    // One captured inner cycle per mask of active instances: a solve changes the mask as instances
    // converge, and the next solve starts from all-active again, so the graphs are kept, not re-captured.
    struct InnerGraph {
        std::vector<int> mask;
        cudaGraphExec_t exec = nullptr;
        int uses = 0, launches = 0;
        std::vector<int> applies;
    };
    std::vector<InnerGraph> graphs;
    double inner_tol = -1.0;
    std::vector<long long> cv;  // operators' configuration generations the graphs were captured with
    std::vector<std::vector<double>> history;
};

static void batch_destroy(BatchWork *b)
{
    if (!b) return;
    if (b->st) cudaStreamSynchronize(b->st);
    for (auto &gr : b->graphs)
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
    for (KrylovWork *k : b->k) kw_free(k);
    if (b->h_pin) cudaFreeHost(b->h_pin);
    for (cudaEvent_t e : b->ev_pull)
        if (e) cudaEventDestroy(e);
    if (b->d_stage) cudaFree(b->d_stage);
    delete b;
}

int batch_create(IeOp *const *ops, int n, int mo, int mi, int precision, void **out)
{
    *out = nullptr;
    if (n < 1) return G2_ERR_ARG;
    if (mo < 1 || mi < 1 || mo > KMAX - 1 || mi > KMAX - 1) {
        g2_set_error_msg("FGMRES buffer sizes must be in [1, 31]");
        return G2_ERR_UNSUPPORTED;
    }
    if (precision < 0 || precision > 1) return G2_ERR_ARG;
    BatchWork *b = new BatchWork();
    b->n = n;
    b->mo = mo;
    b->mi = mi;
    b->precision = precision;
    b->st = ops[0]->stream;
    for (int i = 0; i < n; i++) {
        if (!ops[i]) { batch_destroy(b); return G2_ERR_ARG; }
        b->ops.push_back(ops[i]);
        KrylovWork *k = new KrylovWork();
        b->k.push_back(k);
        const int rc = kw_alloc(k, ops[i]->nvec(), mo, mi, precision);
        if (rc) { batch_destroy(b); return rc; }
    }
    for (int i = 0; i < n;) {
        BatchGroup g;
        g.op = ops[i];
        g.first = i;
        g.n = (i + 1 < n && ops[i + 1] == ops[i]) ? 2 : 1;
        b->groups.push_back(g);
        i += g.n;
    }
    b->h_active.assign(n, 1);
    b->history.resize(n);
    *out = b;
    return G2_OK;
}

void batch_free(void *h) { batch_destroy(reinterpret_cast<BatchWork *>(h)); }

int batch_history(void *h, int i, double *out, int max_len)
{
    BatchWork *b = reinterpret_cast<BatchWork *>(h);
    if (!b || i < 0 || i >= b->n) return 0;
    const int m = (int)b->history[i].size() < max_len ? (int)b->history[i].size() : max_len;
    for (int j = 0; j < m; j++) out[j] = b->history[i][j];
    return m;
}

// applies of the inner level: in_i -> out_i for every instance, paired where two instances share an
// operator (complex64); flag selects the gate of the single applies (F_SOLVER or F_KRYLOV)
template <typename CI, typename FIn, typename FOut>
static int batch_apply(BatchWork *b, FIn in, FOut out, int flag, cudaStream_t st, const BatchGroup *only = nullptr)
{
    for (const BatchGroup &g : b->groups) {
        if (only && &g != only) continue;
        const bool both = g.n == 2 && b->h_active[g.first] && b->h_active[g.first + 1];
        if (both && sizeof(CI) == sizeof(float2)) {
            float2 *U1 = nullptr, *Uh = nullptr;
            int rc = ie_pair_scratch(g.op, &U1, &Uh);
            if (rc) return rc;
            rc = ie_apply_pair32(g.op, reinterpret_cast<const float2 *>(in(g.first)),
                                 reinterpret_cast<const float2 *>(in(g.first + 1)),
                                 reinterpret_cast<float2 *>(out(g.first)), reinterpret_cast<float2 *>(out(g.first + 1)),
                                 st, U1, Uh);
            if (rc == G2_OK) {
                b->k[g.first]->applies32++;
                b->k[g.first + 1]->applies32++;
                continue;
            }
            if (rc != G2_ERR_UNSUPPORTED) return rc;
        }
        for (int i = g.first; i < g.first + g.n; i++) {
            if (!b->h_active[i]) continue;
            const int rc = apply_prec<CI>(g.op, in(i), out(i), st, b->k[i]->Li.flags + flag);
            if (rc) return rc;
            if (sizeof(CI) == sizeof(float2)) b->k[i]->applies32++;
            else b->k[i]->applies64++;
        }
    }
    return G2_OK;
}

// one inner GMRES cycle (x0 = b = v) for every instance: the lockstep form of inner_solve
template <typename CI>
static int batch_inner(BatchWork *b, double tol, cudaStream_t st)
{
    const int n = b->n;
    for (int i = 0; i < n; i++) {
        if (!b->h_active[i]) continue;
        KrylovWork *k = b->k[i];
        Level &L = k->Li;
        const int g = vec_grid(k->N);
        k_zero_level<<<1, 256, 0, st>>>(L); g2_count_launches(1);
        norm2<CI>(k, reinterpret_cast<const CI *>(k->vin), L.scal + S_NRM2, nullptr, st);
        k_set_bn_masked<<<1, 1, 0, st>>>(L, k->Lo.flags + F_KRYLOV); g2_count_launches(1);
        k_copy_or_zero<CI><<<g, kVT, 0, st>>>(reinterpret_cast<CI *>(k->xin), reinterpret_cast<const CI *>(k->vin),
                                             L.scal, k->N); g2_count_launches(1);
    }
    auto vin = [&](int i) { return reinterpret_cast<const CI *>(b->k[i]->vin); };
    auto ri = [&](int i) { return reinterpret_cast<CI *>(b->k[i]->ri); };
    int rc = batch_apply<CI>(b, vin, ri, F_SOLVER, st);
    if (rc) return rc;
    for (int i = 0; i < n; i++) {
        if (!b->h_active[i]) continue;
        KrylovWork *k = b->k[i];
        Level &L = k->Li;
        const int g = vec_grid(k->N);
        const int *solver = L.flags + F_SOLVER;
        CI *r = reinterpret_cast<CI *>(k->ri);
        k_axpby<CI, CI, CI><<<g, kVT, 0, st>>>(r, 1.0, reinterpret_cast<const CI *>(k->vin), -1.0, r, k->N, solver); g2_count_launches(1);
        norm2<CI>(k, r, L.scal + S_NRM2, solver, st);
        k_set_beta<<<1, 1, 0, st>>>(L, tol); g2_count_launches(1);
        k_cycle_start<<<1, 1, 0, st>>>(L, solver); g2_count_launches(1);
        k_scale_by<CI><<<g, kVT, 0, st>>>(reinterpret_cast<CI *>(k->Vi), r, L.scal, S_BETA, k->N, solver); g2_count_launches(1);
    }
    // Arnoldi step j of the active instances in `act`: runs of up to KMI instances with the same vector length
    // share each launch (each instance keeps its own blocks, partials and gates)
    auto arnoldi_step = [&](const std::vector<int> &act, int j) {
        for (size_t c = 0; c < act.size();) {
            KrylovWork *k0 = b->k[act[c]];
            size_t e = c + 1;
            while (e < act.size() && e - c < (size_t)KMI && b->k[act[e]]->N == k0->N && b->k[act[e]]->nparts == k0->nparts)
                e++;
            if (e - c == 1) {
                Level &L = k0->Li;
                CI *Vi = reinterpret_cast<CI *>(k0->Vi);
                cgs<CI>(k0, L, Vi, j, reinterpret_cast<CI *>(k0->wi), L.flags + F_KRYLOV, st);
                arnoldi_tail<CI>(k0, L, Vi, j, reinterpret_cast<const CI *>(k0->wi), tol, L.flags + F_KRYLOV, st);
            } else {
                Multi<CI> mm{};
                for (size_t q = 0; q < e - c; q++) {
                    KrylovWork *k = b->k[act[c + q]];
                    mm.V[q] = reinterpret_cast<CI *>(k->Vi);
                    mm.w[q] = reinterpret_cast<CI *>(k->wi);
                    mm.part[q] = k->part;
                    mm.L[q] = k->Li;
                    mm.gate[q] = k->Li.flags + F_KRYLOV;
                }
                cgs_multi<CI>(mm, (int)(e - c), k0->N, k0->nparts, j, st);
                arnoldi_tail_multi<CI>(mm, (int)(e - c), k0->N, j, tol, st);
            }
            c = e;
        }
    };
    // Each operator group (one frequency's polarisations) runs its apply and then its Arnoldi step before the
    // next group's apply, so the group's fresh w is still in L2 when its Gram-Schmidt reads it (with all
    // applies first, a 16-instance sweep re-read every w from DRAM).  Per instance the sequence of kernels is
    // unchanged.
    for (int j = 0; j < b->mi; j++) {
        auto vj = [&](int i) { return reinterpret_cast<const CI *>(b->k[i]->Vi) + (size_t)j * b->k[i]->N; };
        auto wi = [&](int i) { return reinterpret_cast<CI *>(b->k[i]->wi); };
        for (const BatchGroup &g : b->groups) {
            std::vector<int> act;
            for (int i = g.first; i < g.first + g.n; i++)
                if (b->h_active[i]) act.push_back(i);
            if (act.empty()) continue;
            if ((rc = batch_apply<CI>(b, vj, wi, F_KRYLOV, st, &g))) return rc;
            arnoldi_step(act, j);
        }
    }
    for (int i = 0; i < n; i++) {
        if (!b->h_active[i]) continue;
        KrylovWork *k = b->k[i];
        Level &L = k->Li;
        const int g = vec_grid(k->N);
        const int *solver = L.flags + F_SOLVER;
        CI *x = reinterpret_cast<CI *>(k->xin);
        k_trisolve<<<1, kTriThreads, 0, st>>>(L, solver); g2_count_launches(1);
        k_lincomb<CI, CI><<<g, kVT, 0, st>>>(x, 1.0, x, reinterpret_cast<const CI *>(k->Vi), k->N, L.y, L.flags + F_L,
                                             k->N, solver); g2_count_launches(1);
    }
    return G2_OK;
}

// the inner cycle of all instances: eager on first use, then one captured graph replayed
template <typename CI>
static int batch_inner_fixed(BatchWork *b, double tol, cudaStream_t st)
{
    std::vector<long long> cv;
    for (IeOp *op : b->ops) cv.push_back(op->config_gen);
    const char *ng = std::getenv("GIEM2G_NO_GRAPHS");
    const bool use_graphs = !(ng && ng[0] == '1');
    if (b->inner_tol != tol || b->cv != cv) {  // the captured arguments are stale: drop every graph
        for (auto &gr : b->graphs)
            if (gr.exec) cudaGraphExecDestroy(gr.exec);
        b->graphs.clear();
        b->inner_tol = tol;
        b->cv = cv;
    }
    BatchWork::InnerGraph *gr = nullptr;
    for (auto &e : b->graphs)
        if (e.mask == b->h_active) gr = &e;
    if (!gr) {
        constexpr size_t kMaxGraphs = 32;
        if (b->graphs.size() >= kMaxGraphs) {  // oldest first
            if (b->graphs.front().exec) cudaGraphExecDestroy(b->graphs.front().exec);
            b->graphs.erase(b->graphs.begin());
        }
        b->graphs.emplace_back();
        gr = &b->graphs.back();
        gr->mask = b->h_active;
        gr->applies.assign(b->n, 0);
    }
    auto credit = [&]() {
        g2_count_launches(gr->launches);
        for (int i = 0; i < b->n; i++) {
            if (sizeof(CI) == sizeof(float2)) b->k[i]->applies32 += gr->applies[i];
            else b->k[i]->applies64 += gr->applies[i];
        }
    };
    if (gr->exec) {
        G2_CUDA_CHECK(cudaGraphLaunch(gr->exec, st));
        credit();
        return G2_OK;
    }
    // first use of a mask runs eagerly (it may allocate pair scratch, which a capture cannot)
    if (!use_graphs || gr->uses++ == 0) return batch_inner<CI>(b, tol, st);
    std::vector<int> a0(b->n);
    for (int i = 0; i < b->n; i++) a0[i] = b->k[i]->applies32 + b->k[i]->applies64;
    const long long l0 = g2_launch_total();
    cudaGraph_t graph = nullptr;
    G2_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int rc = batch_inner<CI>(b, tol, st);
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (rc) return rc;
    if (ce != cudaSuccess) {
        g2_set_error(__FILE__, __LINE__, cudaGetErrorString(ce));
        return G2_ERR_CUDA;
    }
    gr->launches = (int)(g2_launch_total() - l0);
    for (int i = 0; i < b->n; i++) {
        KrylovWork *k = b->k[i];
        gr->applies[i] = k->applies32 + k->applies64 - a0[i];
        if (sizeof(CI) == sizeof(float2)) k->applies32 -= gr->applies[i];
        else k->applies64 -= gr->applies[i];
    }
    ce = cudaGraphInstantiate(&gr->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
        g2_set_error(__FILE__, __LINE__, cudaGetErrorString(ce));
        gr->exec = nullptr;
        return G2_ERR_CUDA;
    }
    G2_CUDA_CHECK(cudaGraphLaunch(gr->exec, st));
    credit();
    return G2_OK;
}

// per-instance host copies of the outer level's scalars and flags, one synchronisation for all
struct BatchScal {
    double s[S_NSCAL];
    int f[F_NFLAGS];
};
// Copies of the outer level's scalars and flags of instances `which` into pinned slot `slot` (pageable
// destinations made every such read a staged, blocking copy), completed by the slot's event.
static int batch_pull_start(BatchWork *b, const std::vector<int> &which, int slot, cudaStream_t st)
{
    if (!b->h_pin) {
        G2_CUDA_CHECK(cudaMallocHost(&b->h_pin, 2 * sizeof(BatchScal) * b->n));
        for (cudaEvent_t &e : b->ev_pull) G2_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    BatchScal *h = reinterpret_cast<BatchScal *>(b->h_pin) + (size_t)slot * b->n;
    for (int i : which) {
        G2_CUDA_CHECK(cudaMemcpyAsync(h[i].s, b->k[i]->Lo.scal, sizeof(h[i].s), cudaMemcpyDeviceToHost, st));
        G2_CUDA_CHECK(cudaMemcpyAsync(h[i].f, b->k[i]->Lo.flags, sizeof(h[i].f), cudaMemcpyDeviceToHost, st));
    }
    G2_CUDA_CHECK(cudaEventRecord(b->ev_pull[slot], st));
    return G2_OK;
}
static int batch_pull_finish(BatchWork *b, const std::vector<int> &which, int slot, std::vector<BatchScal> &h)
{
    G2_CUDA_CHECK(cudaEventSynchronize(b->ev_pull[slot]));
    const BatchScal *p = reinterpret_cast<const BatchScal *>(b->h_pin) + (size_t)slot * b->n;
    for (int i : which) h[i] = p[i];
    return G2_OK;
}
static std::vector<int> active_list(const BatchWork *b)
{
    std::vector<int> a;
    for (int i = 0; i < b->n; i++)
        if (b->h_active[i]) a.push_back(i);
    return a;
}
// per-instance host copies of the active instances' scalars and flags, one synchronisation for all
static int batch_pull(BatchWork *b, std::vector<BatchScal> &h, cudaStream_t st)
{
    const std::vector<int> act = active_list(b);
    int rc = batch_pull_start(b, act, 0, st);
    if (!rc) rc = batch_pull_finish(b, act, 0, h);
    if (rc) return rc;
    for (IeOp *op : b->ops) {
        const int e = ie_check_device_error(op);
        if (e) return e;
    }
    return G2_OK;
}

// The same copies into pinned slot `slot` without waiting, so the host can enqueue more work before it waits
// (batch_outer's outer step j + 1).
static int batch_pull_async(BatchWork *b, int slot, cudaStream_t st)
{
    return batch_pull_start(b, active_list(b), slot, st);
}
static int batch_pull_wait(BatchWork *b, int slot, std::vector<BatchScal> &h)
{
    return batch_pull_finish(b, active_list(b), slot, h);
}

// FinalActions of instance i (gmres.F90:382-421) after the host learned that it stops
template <typename CI>
static void batch_final_launch(BatchWork *b, int i, cudaStream_t st, int &rc)
{
    KrylovWork *k = b->k[i];
    Level &L = k->Lo;
    const int g = vec_grid(k->N);
    CI *Z = reinterpret_cast<CI *>(k->Zo);
    k_trisolve<<<1, kTriThreads, 0, st>>>(L, nullptr); g2_count_launches(1);
    k_lincomb<double2, CI><<<g, kVT, 0, st>>>(k->x, 1.0, k->x, Z, k->N, L.y, L.flags + F_L, k->N, nullptr); g2_count_launches(1);
    if ((rc = ie_apply_device64(b->ops[i], k->x, k->r0, st))) return;
    k->applies64++;
    k_axpby<double2, double2, double2><<<g, kVT, 0, st>>>(k->r0, 1.0, k->b, -1.0, k->r0, k->N, nullptr); g2_count_launches(1);
    norm2<double2>(k, k->r0, L.scal + S_NRM2, nullptr, st);
}

template <typename CI>
static int batch_outer(BatchWork *b, const GIEM2G_FGMRES_CTL &ctl, GIEM2G_RESULT *info, cudaStream_t st)
{
    const int n = b->n, M = b->mo;
    const double tol = ctl.misfit;
    std::vector<BatchScal> h(n);
    std::vector<double> bn(n, 0.0), bea(n, -1.0);
    std::vector<int> iter(n, 0), converged(n, 0), finishing(n, 0);
    int rc = G2_OK;
    char msg[256];
    for (int i = 0; i < n; i++) {
        b->history[i].clear();
        b->h_active[i] = 1;
        info[i].iterations = 0;
        info[i].bea = -1.0;
        info[i].be = -1.0;
        info[i].stat = -1;
    }
    // gmres.F90:129-168 for every instance, with one host read: the initial residual is gated on the device
    // flag k_set_bn clears for a zero right-hand side, so the host need not read ||b|| before launching it
    for (int i = 0; i < n; i++) {
        KrylovWork *k = b->k[i];
        const int g = vec_grid(k->N);
        const int *solver = k->Lo.flags + F_SOLVER;
        k_zero_level<<<1, 256, 0, st>>>(k->Lo); g2_count_launches(1);
        norm2<double2>(k, k->b, k->Lo.scal + S_NRM2, nullptr, st);
        k_set_bn<<<1, 1, 0, st>>>(k->Lo); g2_count_launches(1);
        if ((rc = ie_apply_device64(b->ops[i], k->x, k->r0, st, solver))) return rc;
        k_axpby<double2, double2, double2><<<g, kVT, 0, st>>>(k->r0, 1.0, k->b, -1.0, k->r0, k->N, solver); g2_count_launches(1);
        k_axpby<double2, double2, double2><<<g, kVT, 0, st>>>(k->w, 1.0, k->r0, 0.0, (const double2 *)nullptr, k->N, solver); g2_count_launches(1);
        norm2<double2>(k, k->w, k->Lo.scal + S_NRM2, solver, st);
        k_set_beta<<<1, 1, 0, st>>>(k->Lo, tol); g2_count_launches(1);
    }
    if ((rc = batch_pull(b, h, st))) return rc;
    for (int i = 0; i < n; i++) {
        KrylovWork *k = b->k[i];
        bn[i] = h[i].s[S_BN];
        if (bn[i] < ZERO_THRESHOLD) {
            cudaMemsetAsync(k->x, 0, sizeof(double2) * k->N, st);
            info[i].stat = 1;
            b->h_active[i] = 0;
            continue;
        }
        k->applies64++;
    }
    for (int i = 0; i < n; i++) {
        if (!b->h_active[i]) continue;
        if (h[i].s[S_BETA] / bn[i] < tol) {
            info[i].stat = 1;
            info[i].be = h[i].s[S_BETA] / bn[i];
            b->h_active[i] = 0;
        }
    }
    auto any_active = [&]() {
        for (int i = 0; i < n; i++)
            if (b->h_active[i]) return true;
        return false;
    };
    while (any_active()) {
        for (int i = 0; i < n; i++) {
            if (!b->h_active[i]) continue;
            KrylovWork *k = b->k[i];
            k_cycle_start<<<1, 1, 0, st>>>(k->Lo, nullptr); g2_count_launches(1);
            k_scale_by<double2><<<vec_grid(k->N), kVT, 0, st>>>(k->Vo, k->w, k->Lo.scal, S_BETA, k->N, nullptr); g2_count_launches(1);
        }
        bool cycle_done = false;
        // Outer step j of every active instance.  Its kernels are gated by the instance's outer Krylov flag,
        // which the Arnoldi tail of step j - 1 clears when the instance converged (or its cycle ended): step
        // j + 1 is enqueued before the host reads step j's misfits, so the GPU does not wait for the host
        // between steps, and an instance that converged at step j does nothing in step j + 1.  The arithmetic
        // of the instances that go on is unchanged.
        auto enqueue_step = [&](int j) -> int {
            for (int i = 0; i < n; i++) {
                if (!b->h_active[i]) continue;
                KrylovWork *k = b->k[i];
                const int *go = k->Lo.flags + F_KRYLOV;
                k_axpby<CI, double2, double2><<<vec_grid(k->N), kVT, 0, st>>>(
                    reinterpret_cast<CI *>(k->vin), 1.0, k->Vo + (size_t)j * k->N, 0.0, (const double2 *)nullptr, k->N,
                    go); g2_count_launches(1);
            }
            int r = batch_inner_fixed<CI>(b, tol, st);
            if (r) return r;
            // per operator group: the FP64 applies, then the group's outer Arnoldi step (w still in L2), with
            // the group's instances sharing each CGS and scaling launch
            for (const BatchGroup &gr : b->groups) {
                std::vector<int> act;
                for (int i = gr.first; i < gr.first + gr.n; i++) {
                    if (!b->h_active[i]) continue;
                    act.push_back(i);
                    KrylovWork *k = b->k[i];
                    const int g = vec_grid(k->N);
                    const int *go = k->Lo.flags + F_KRYLOV;
                    CI *Zj = reinterpret_cast<CI *>(k->Zo) + (size_t)j * k->N;
                    k_axpby<CI, CI, CI><<<g, kVT, 0, st>>>(Zj, 1.0, reinterpret_cast<const CI *>(k->xin), 0.0, (const CI *)nullptr, k->N, go); g2_count_launches(1);
                    if (sizeof(CI) == sizeof(double2)) {
                        if ((r = ie_apply_device64(b->ops[i], reinterpret_cast<const double2 *>(Zj), k->w, st, go))) return r;
                    } else {
                        k_axpby<double2, CI, CI><<<g, kVT, 0, st>>>(k->tmp, 1.0, Zj, 0.0, (const CI *)nullptr, k->N, go); g2_count_launches(1);
                        if ((r = ie_apply_device64(b->ops[i], k->tmp, k->w, st, go))) return r;
                    }
                }
                if (act.size() == 1) {
                    KrylovWork *k0 = b->k[act[0]];
                    const int *go = k0->Lo.flags + F_KRYLOV;
                    cgs<double2>(k0, k0->Lo, k0->Vo, j, k0->w, go, st);
                    arnoldi_tail<double2>(k0, k0->Lo, k0->Vo, j, k0->w, tol, go, st);
                } else if (act.size() == 2 && b->k[act[0]]->N == b->k[act[1]]->N &&
                           b->k[act[0]]->nparts == b->k[act[1]]->nparts) {
                    Multi<double2> mm{};
                    for (size_t q = 0; q < act.size(); q++) {
                        KrylovWork *k = b->k[act[q]];
                        mm.V[q] = k->Vo;
                        mm.w[q] = k->w;
                        mm.part[q] = k->part;
                        mm.L[q] = k->Lo;
                        mm.gate[q] = k->Lo.flags + F_KRYLOV;
                    }
                    cgs_multi<double2>(mm, 2, b->k[act[0]]->N, b->k[act[0]]->nparts, j, st);
                    arnoldi_tail_multi<double2>(mm, 2, b->k[act[0]]->N, j, tol, st);
                } else {
                    for (int i : act) {
                        KrylovWork *k = b->k[i];
                        const int *go = k->Lo.flags + F_KRYLOV;
                        cgs<double2>(k, k->Lo, k->Vo, j, k->w, go, st);
                        arnoldi_tail<double2>(k, k->Lo, k->Vo, j, k->w, tol, go, st);
                    }
                }
            }
            return G2_OK;
        };
        // Running ahead is skipped when an instance is expected to converge at step j (its last misfit times
        // its last reduction factor within kAheadMargin of the tolerance): a step enqueued after that keeps the
        // pair's shared complex64 applies for an instance that would otherwise run its single applies.
        auto near_tol = [&]() {
            constexpr double kAheadMargin = 4.0;
            for (int i = 0; i < n; i++) {
                if (!b->h_active[i] || b->history[i].empty()) continue;
                const std::vector<double> &hs = b->history[i];
                const double last = hs.back();
                const double r = hs.size() > 1 && hs[hs.size() - 2] > 0.0 ? std::min(1.0, last / hs[hs.size() - 2]) : 1.0;
                if (last * r < kAheadMargin * tol) return true;
            }
            return false;
        };
        bool ahead = false;  // step j was enqueued ahead, during step j - 1
        for (int j = 0; j < M && !cycle_done; j++) {
            if (!ahead && (rc = enqueue_step(j))) return rc;
            if ((rc = batch_pull_async(b, j & 1, st))) return rc;
            ahead = j + 1 < M && !near_tol();
            if (ahead && (rc = enqueue_step(j + 1))) return rc;
            if ((rc = batch_pull_wait(b, j & 1, h))) return rc;
            // an instance still active here ran step j (it had not converged at step j - 1)
            for (int i = 0; i < n; i++)
                if (b->h_active[i]) b->k[i]->applies64++;
            for (int i = 0; i < n; i++) {
                if (!b->h_active[i]) continue;
                bea[i] = h[i].s[S_BEA];
                if (!std::isfinite(bea[i])) {
                    g2_set_error_msg("FGMRES: non-finite Arnoldi misfit");
                    return G2_ERR_NUMERIC;
                }
                b->history[i].push_back(bea[i]);
                std::snprintf(msg, sizeof(msg), "FGMRES outer  iteration:%5d Arnoldy misfit: %10.3E  (instance %d)",
                              (int)b->history[i].size(), bea[i], i);
                g2_log(msg);
                if (bea[i] < tol) {
                    converged[i] = 1;
                    finishing[i] = 1;
                    b->h_active[i] = 0;
                }
            }
            if (!any_active()) cycle_done = true;
        }
        // end of the cycle for the instances still running: restart or give up (gmres.F90:186-212)
        for (int i = 0; i < n; i++) {
            if (!b->h_active[i]) continue;
            KrylovWork *k = b->k[i];
            const int g = vec_grid(k->N);
            iter[i]++;
            if (iter[i] >= ctl.fgmres_maxit) {
                finishing[i] = 1;
                b->h_active[i] = 0;
                continue;
            }
            k_trisolve<<<1, kTriThreads, 0, st>>>(k->Lo, nullptr); g2_count_launches(1);
            k_lincomb<double2, CI><<<g, kVT, 0, st>>>(k->x, 1.0, k->x, reinterpret_cast<const CI *>(k->Zo), k->N,
                                                      k->Lo.y, k->Lo.flags + F_L, k->N, nullptr); g2_count_launches(1);
            k_restart_g<<<1, 1, 0, st>>>(k->Lo); g2_count_launches(1);
            k_copy_g<<<1, 64, 0, st>>>(k->Lo); g2_count_launches(1);
            k_lincomb<double2, double2><<<g, kVT, 0, st>>>(k->w, 0.0, (const double2 *)nullptr, k->Vo, k->N, k->Lo.y,
                                                           k->Lo.flags + F_L, k->N, nullptr); g2_count_launches(1);
        }
        // instances that stopped in this cycle: final actions now (their own kernels only)
        for (int i = 0; i < n; i++) {
            if (!finishing[i]) continue;
            batch_final_launch<CI>(b, i, st, rc);
            if (rc) return rc;
        }
        bool any_fin = false;
        for (int i = 0; i < n; i++) any_fin = any_fin || finishing[i];
        if (any_fin) {
            // read the true residuals of the instances that finished (pull reads active ones only)
            std::vector<int> fin;
            for (int i = 0; i < n; i++)
                if (finishing[i]) fin.push_back(i);
            if ((rc = batch_pull_start(b, fin, 0, st)) || (rc = batch_pull_finish(b, fin, 0, h))) return rc;
            for (int i = 0; i < n; i++) {
                if (!finishing[i]) continue;
                const double be = std::sqrt(h[i].s[S_NRM2]) / bn[i];
                info[i].iterations = (int)b->history[i].size();
                info[i].bea = bea[i];
                info[i].be = be;
                info[i].stat = converged[i] ? (be >= tol ? 2 : 1) : -1;
                finishing[i] = 0;
            }
        }
    }
    return G2_OK;
}

int batch_solve_device(void *h, const double2 *const *d_Ebkg, double2 *const *d_Esol, const double2 *const *d_E0,
                       const GIEM2G_FGMRES_CTL &ctl, GIEM2G_RESULT *info)
{
    BatchWork *b = reinterpret_cast<BatchWork *>(h);
    if (!b) return G2_ERR_STATE;
    if (ctl.fgmres_buf != b->mo || ctl.gmres_buf != b->mi || (ctl.precision >= 0 && ctl.precision != b->precision)) {
        g2_set_error_msg("batched solve: buffer sizes or precision differ from the batch's");
        return G2_ERR_ARG;
    }
    cudaStream_t st = b->st;
    for (IeOp *op : b->ops)
        if (op->stream != st) G2_CUDA_CHECK(cudaStreamSynchronize(op->stream));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    for (int i = 0; i < b->n; i++) {
        IeOp *op = b->ops[i];
        KrylovWork *k = b->k[i];
        k->applies32 = k->applies64 = 0;
        const int g = vec_grid(k->N);
        // SolveEquation (ie_solver_module.F90:62-80): rhs = sqrt(Re sb) E_bkg; guess = E0/a or rhs
        k_rhs<<<g, 256, 0, st>>>(k->b, d_Ebkg[i], op->d_post64, (size_t)op->Nx * op->Ny, op->Nz); g2_count_launches(1);
        if (d_E0 && d_E0[i]) {
            k_scale_asig<<<g, 256, 0, st>>>(k->x, d_E0[i], op->d_asig64, op->cells(), true); g2_count_launches(1);
        } else {
            G2_CUDA_CHECK(cudaMemcpyAsync(k->x, k->b, sizeof(double2) * k->N, cudaMemcpyDeviceToDevice, st));
        }
    }
    int rc = b->precision == 0 ? batch_outer<double2>(b, ctl, info, st) : batch_outer<float2>(b, ctl, info, st);
    if (rc) return rc;
    for (int i = 0; i < b->n; i++) {
        IeOp *op = b->ops[i];
        KrylovWork *k = b->k[i];
        k_scale_asig<<<vec_grid(k->N), 256, 0, st>>>(d_Esol[i], k->x, op->d_asig64, op->cells(), false); g2_count_launches(1);
    }
    cudaEventRecord(e1, st);
    G2_CUDA_CHECK(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (int i = 0; i < b->n; i++) {
        info[i].applies_fp64 = b->k[i]->applies64;
        info[i].applies_fp32 = b->k[i]->applies32;
        info[i].device_ms = ms;
        b->ops[i]->mult_num += b->k[i]->applies64 + b->k[i]->applies32;
    }
    for (IeOp *op : b->ops) {
        const int e = ie_check_device_error(op);
        if (e) return e;
    }
    return G2_OK;
}

int batch_stage(void *h, double2 **d_stage, size_t *N)
{
    BatchWork *b = reinterpret_cast<BatchWork *>(h);
    if (!b) return G2_ERR_STATE;
    size_t nmax = 0;
    for (IeOp *op : b->ops) nmax = op->nvec() > nmax ? op->nvec() : nmax;
    if (!b->d_stage) G2_CUDA_CHECK(cudaMalloc(&b->d_stage, sizeof(double2) * nmax * 3 * b->n));
    *d_stage = b->d_stage;
    *N = nmax;
    return G2_OK;
}

int batch_size(void *h) { return h ? reinterpret_cast<BatchWork *>(h)->n : 0; }
IeOp *batch_op(void *h, int i) { return reinterpret_cast<BatchWork *>(h)->ops[i]; }
