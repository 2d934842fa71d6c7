// IE operator apply on one GPU: y = sqrt(Re sb) * (a*x - IDFT2[ G_hat . DFT2(gsig*x) ] / (dz*4NxNy))
//
// Restates APPLY_PRECOND / MULT_IE_OP (apply_ie_operator_module.F90:39-263) without the MPI
// slab decomposition: the padded 2Nx x 2Ny transform of the reference's Distributed_FFT.F90
// becomes five kernels over HBM-resident buffers:
//   k_fx       pre-scale by gsig, zero-pad in x, forward x-FFT          x   -> U1[kx][y][zc]
//   k_fy       zero-pad in y, forward y-FFT, scatter to (q,r,slot)      U1  -> Uhat[q][r][4][zc]
//   contraction per (q,r): 6 Green's blocks applied to the 4 points (+-kx,+-ky)   Uhat in place
//              (contract.cu, TMA-pipelined; k_contract below is the generic fallback)
//   k_by       inverse y-FFT, crop y<Ny                                 Uhat -> U1
//   k_bx       inverse x-FFT, crop x<Nx, post-combine                   U1  -> y
// The transforms are four-step register FFTs (fft4.cuh) with one shared-memory transpose; zc = c*Nz+z
// is the fastest index of the intermediates so every global access is coalesced.
// (kx-pair q, ky-pair r, slot s) <-> (kx,ky): kx = q (s&2==0) or 2Nx-q, with q=0,s&2 the x-Nyquist;
// ky = r (s&1==0) or 2Ny-r, with r=0,s&1 the y-Nyquist.  Nyquist outputs are zero as in the
// reference (FinalTransposeRepack / DistributedFourierYRepack drop them).
#include <algorithm>
#include <type_traits>
#include "common.cuh"
#include "fft4.cuh"
#include "ie_internal.h"

namespace {

template <typename R> using CT = typename Cplx<R>::T;

constexpr int kThreads = 256;

// Launch bounds of the FFT passes.  CAP = 0: any block up to 256 threads, registers as the compiler likes
// (100-130 in FP64, 90-100 in complex64 at 2Ny = 256).  CAP = 1 holds more blocks per SM -- the passes are
// latency-bound at 14-16 resident warps: complex64 at 64 registers (4 blocks of 256 threads), FP64 at 128
// (4 blocks of 128 threads, so only for 8 lines per CTA).  Measured per apply at 128x128x32: complex64 passes
// 88 -> 77 us, FP64 139 -> 128 us; tighter caps spill and lose (FP64 at 96 registers, 5 blocks: k_fx spilled
// 36 bytes and the whole FP64 apply took 0.320 against 0.312 ms).  Used for 2Ny, 2Nx <= 256 (the larger
// register DFTs of longer lines do not fit the caps).
template <typename R, int CAP> struct PassLB { static constexpr int T = kThreads, B = 1; };
template <> struct PassLB<float, 1> { static constexpr int T = 256, B = 4; };
template <> struct PassLB<double, 1> { static constexpr int T = 128, B = 4; };

// The vectors of one apply: nv = 1, or nv = 2 right-hand sides of the same operator that share every
// tensor read.  Line zc of a pass runs over [0, nv*3Nz): vector zc / 3Nz, row zc % 3Nz.
template <typename C> struct VecSet {
    const C *in[2];
    C *out[2];
    int nv;
};

// slot helpers: (kx-pair q, slot bit) and (ky-pair r, mirror bit) of a spectral index
G2_D void kx_to_slot(int kx, int Nx, int &q, int &sx)
{
    if (kx < Nx) { q = kx; sx = 0; }
    else if (kx == Nx) { q = 0; sx = 1; }
    else { q = 2 * Nx - kx; sx = 1; }
}
G2_D void ky_to_slot(int ky, int Ny, int &r, int &sy)
{
    if (ky < Ny) { r = ky; sy = 0; }
    else if (ky == Ny) { r = 0; sy = 1; }
    else { r = 2 * Ny - ky; sy = 1; }
}

template <typename C>
G2_D void load_tw(C *dst, const C *__restrict__ src, int L)
{
    for (int i = threadIdx.x; i < L; i += blockDim.x) dst[i] = src[i];
}

// ---------------------------------------------------------------------------------------------
// k_fx: pre-scale by gsig, zero-pad to 2Nx, forward x-FFT.  CTA = one y row x NL (z,c) lines.
// apply_ie_operator_module.F90:57-115 + Distributed_FFT.F90:552-569
template <typename R, int L, int CAP>
__global__ void __launch_bounds__(PassLB<R, CAP>::T, PassLB<R, CAP>::B) k_fx(const VecSet<CT<R>> vs, const CT<R> *__restrict__ gsig,
                                                 CT<R> *__restrict__ U1, const CT<R> *__restrict__ twg, int Nx,
                                                 int Ny, int Nz, int NL, const int *gate)
{
    if (gate && *gate == 0) return;
    using C = CT<R>;
    constexpr int N1 = Fact<L>::N1, N2 = Fact<L>::N2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *sm = tw + L;
    // indices fit 32 bits: every buffer holds fewer than 2^31 elements for 2Nx, 2Ny <= 1024
    const int Z3 = 3 * Nz, ZL = vs.nv * Z3, zc0 = blockIdx.x * NL, y = blockIdx.y;
    const int nl = min(NL, ZL - zc0);
    const int plane = Nx * Ny, row = y * Nx;
    load_tw(tw, twg, L);
    __syncthreads();
    auto load = [&](int t, int x) -> C {
        const int zc = zc0 + t, v = zc >= Z3 ? 1 : 0, lzc = zc - v * Z3, z = lzc % Nz;
        const C *in = v ? vs.in[1] : vs.in[0];  // select, not index: keeps the parameters out of local memory
        return cmul(in[lzc * plane + row + x], gsig[z * plane + row + x]);
    };
    auto store = [&](int t, int kx, C v) { U1[(kx * Ny + y) * ZL + zc0 + t] = v; };
    auto off = [&](int t, int n1, int k2) { return n1 + N1 * k2 + (L + 1) * t; };
    fft4step<C, N1, N2, false, true, false, false, true>(sm, nl, ilog2(NL), tw, load, store, off);
}

// k_fy: zero-pad to 2Ny, forward y-FFT of one kx column, scatter to (q, r, slot).
// Distributed_FFT.F90:437-505 (y transform + +-ky repack) and :639-694 (+-kx repack)
template <typename R, int L, int CAP>
__global__ void __launch_bounds__(PassLB<R, CAP>::T, PassLB<R, CAP>::B) k_fy(const CT<R> *__restrict__ U1, CT<R> *__restrict__ Uh,
                                                 const CT<R> *__restrict__ twg, int Nx, int Ny, int Nz, int NL,
                                                 int nv, const int *gate)
{
    if (gate && *gate == 0) return;
    using C = CT<R>;
    constexpr int N1 = Fact<L>::N1, N2 = Fact<L>::N2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *sm = tw + L;
    const int Z3 = nv * 3 * Nz, zc0 = blockIdx.x * NL, kx = blockIdx.y;  // Z3: lines of all vectors
    const int nl = min(NL, Z3 - zc0);
    int q, sx;
    kx_to_slot(kx, Nx, q, sx);
    if (kx == Nx) {  // x-Nyquist column: kept zero
        for (int i = threadIdx.x; i < nl * L; i += blockDim.x) {
            const int t = i % nl, ky = i / nl;
            int r, sy;
            ky_to_slot(ky, Ny, r, sy);
            Uh[(((size_t)q * Ny + r) * 4 + sx * 2 + sy) * Z3 + zc0 + t] = czero<C>();
        }
        return;
    }
    load_tw(tw, twg, L);
    __syncthreads();
    const C *col = U1 + kx * Ny * Z3 + zc0;
    C *dst = Uh + q * Ny * 4 * Z3 + sx * 2 * Z3 + zc0;
    auto load = [&](int t, int yy) -> C { return col[yy * Z3 + t]; };
    auto store = [&](int t, int ky, C v) {
        int r, sy;
        ky_to_slot(ky, L / 2, r, sy);  // L = 2Ny: with the output index's range known, this folds per output
        dst[(r * 4 + sy) * Z3 + t] = v;
    };
    auto off = [&](int t, int n1, int k2) { return t + NL * (n1 + N1 * k2); };
    fft4step<C, N1, N2, false, true, false, true, true>(sm, nl, ilog2(NL), tw, load, store, off);
}

// k_by: inverse y-FFT of one kx column, crop y < Ny.  Distributed_FFT.F90:455-476, 696-788
template <typename R, int L, int CAP>
__global__ void __launch_bounds__(PassLB<R, CAP>::T, PassLB<R, CAP>::B) k_by(const CT<R> *__restrict__ Uh, CT<R> *__restrict__ U1,
                                                 const CT<R> *__restrict__ twg, int Nx, int Ny, int Nz, int NL,
                                                 int nv, const int *gate)
{
    if (gate && *gate == 0) return;
    using C = CT<R>;
    constexpr int N1 = Fact<L>::N1, N2 = Fact<L>::N2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *sm = tw + L;
    const int Z3 = nv * 3 * Nz, zc0 = blockIdx.x * NL, kx = blockIdx.y;  // Z3: lines of all vectors
    if (kx == Nx) return;  // x-Nyquist column is read as zero by k_bx
    const int nl = min(NL, Z3 - zc0);
    int q, sx;
    kx_to_slot(kx, Nx, q, sx);
    load_tw(tw, twg, L);
    __syncthreads();
    const C *src = Uh + q * Ny * 4 * Z3 + sx * 2 * Z3 + zc0;
    C *col = U1 + kx * Ny * Z3 + zc0;
    auto load = [&](int t, int ky) -> C {
        int r, sy;
        ky_to_slot(ky, L / 2, r, sy);  // L = 2Ny: folds per input at compile time
        return src[(r * 4 + sy) * Z3 + t];
    };
    auto store = [&](int t, int yy, C v) { col[yy * Z3 + t] = v; };
    auto off = [&](int t, int n1, int k2) { return t + NL * (n1 + N1 * k2); };
    fft4step<C, N1, N2, true, false, true, true, true>(sm, nl, ilog2(NL), tw, load, store, off);
}

// k_bx: inverse x-FFT, crop x < Nx, post-combine y = s*(a*x - w/(dz*4NxNy)).
// apply_ie_operator_module.F90:125-174
template <typename R, int L, int CAP>
__global__ void __launch_bounds__(PassLB<R, CAP>::T, PassLB<R, CAP>::B) k_bx(const CT<R> *__restrict__ U1, const VecSet<CT<R>> vs,
                                                 const CT<R> *__restrict__ asig, const R *__restrict__ post,
                                                 const CT<R> *__restrict__ twg, int Nx, int Ny, int Nz, int NL,
                                                 const int *gate)
{
    if (gate && *gate == 0) return;
    using C = CT<R>;
    constexpr int N1 = Fact<L>::N1, N2 = Fact<L>::N2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *tw = reinterpret_cast<C *>(smem_raw);
    C *sm = tw + L;
    const int Z3 = 3 * Nz, ZL = vs.nv * Z3, zc0 = blockIdx.x * NL, y = blockIdx.y;
    const int nl = min(NL, ZL - zc0);
    const int plane = Nx * Ny, row = y * Nx;
    load_tw(tw, twg, L);
    __syncthreads();
    auto load = [&](int t, int kx) -> C {
        return kx == L / 2 ? czero<C>() : U1[(kx * Ny + y) * ZL + zc0 + t];  // L = 2Nx
    };
    // a*x of each output, read before the inverse transform of its line (see fft4step_pre)
    auto pre = [&](int t, int x) -> C {
        const int zc = zc0 + t, v = zc >= Z3 ? 1 : 0, lzc = zc - v * Z3, z = lzc % Nz;
        const C *in = v ? vs.in[1] : vs.in[0];
        return cmul(in[lzc * plane + row + x], asig[z * plane + row + x]);
    };
    auto store = [&](int t, int x, C w, C d1) {
        const int zc = zc0 + t, v = zc >= Z3 ? 1 : 0, lzc = zc - v * Z3, z = lzc % Nz;
        C *out = v ? vs.out[1] : vs.out[0];
        const R sq = post[z], inv = post[Nz + z];
        C o;
        o.x = (d1.x - w.x * inv) * sq;
        o.y = (d1.y - w.y * inv) * sq;
        out[lzc * plane + row + x] = o;
    };
    auto off = [&](int t, int n1, int k2) { return t * (L + 1) + k2 + N2 * n1; };
    fft4step_pre<C, N1, N2, true, false, true, true, false>(sm, nl, ilog2(NL), tw, load, pre, store, off);
}

// ---------------------------------------------------------------------------------------------
// k_contract: one CTA per (q,r).  apply_ie_operator_module.F90:265-374 (VERTICAL_MULT_GENERAL[_ZERO]).
// Thread t < 3Nz owns output row (c,z) for the 4 points.  Tensor unit in smem:
//   [xx P][xy P][yy P][zz P] packed upper (i<=j -> i + j(j+1)/2), [xz Nz*Nz][yz Nz*Nz] column-major.
// Point signs (sigma_x, m) from slot s: sigma_x = -1 if s&2, m = -1 if s&1:
//   xy: sigma_x*m   xz: sigma_x   zx: -sigma_x (xz^T)   yz: m   zy: -m (yz^T)   diagonal blocks: +1
template <typename R>
__global__ void k_contract(const CT<R> *__restrict__ G, CT<R> *__restrict__ Uhat, int Nx, int Ny, int Nz,
                           const int *gate)
{
    if (gate && *gate == 0) return;
    const int AW = sizeof(R) == 8 ? asw_width64(Nz) : asw_width32(Nz);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int P = Nz * (Nz + 1) / 2, T = 4 * P + 2 * Nz * Nz, Z3 = 3 * Nz;
    CT<R> *sg = reinterpret_cast<CT<R> *>(smem_raw);
    CT<R> *su = sg + T;  // [4][3Nz]
    const size_t unit = blockIdx.x;
    const int q = (int)(unit / Ny), r = (int)(unit - (size_t)q * Ny);
    {
        // 16-byte vector copy of the tensor unit
        const int nbytes = T * (int)sizeof(CT<R>);
        const int4 *src = reinterpret_cast<const int4 *>(G + unit * T);
        int4 *dst = reinterpret_cast<int4 *>(sg);
        // T = 2Nz(2Nz+1) is even, so every unit starts on a 16-byte boundary for both precisions
        for (int i = threadIdx.x; i < nbytes / 16; i += blockDim.x) dst[i] = __ldcs(src + i);
        for (int i = threadIdx.x; i < 4 * Z3; i += blockDim.x) su[i] = Uhat[unit * 4 * Z3 + i];
    }
    __syncthreads();
    const int t = threadIdx.x;
    if (t >= Z3) return;
    const int c = t / Nz, z = t - c * Nz;
    CT<R> acc[4];
#pragma unroll
    for (int p = 0; p < 4; p++) acc[p] = czero<CT<R>>();
    for (int cp = 0; cp < 3; cp++) {
        CT<R> part[4];
#pragma unroll
        for (int p = 0; p < 4; p++) part[p] = czero<CT<R>>();
        // block selection
        int kind;  // 0: symmetric packed, 1: asym (z,z'), 2: asym transposed (z',z)
        const CT<R> *blk;
        if (c == 0 && cp == 0) { kind = 0; blk = sg + 0 * P; }
        else if ((c == 0 && cp == 1) || (c == 1 && cp == 0)) { kind = 0; blk = sg + 1 * P; }
        else if (c == 1 && cp == 1) { kind = 0; blk = sg + 2 * P; }
        else if (c == 2 && cp == 2) { kind = 0; blk = sg + 3 * P; }
        else if (c == 0 && cp == 2) { kind = 1; blk = sg + 4 * P; }
        else if (c == 1 && cp == 2) { kind = 1; blk = sg + 4 * P + Nz * Nz; }
        else if (c == 2 && cp == 0) { kind = 2; blk = sg + 4 * P; }
        else { kind = 2; blk = sg + 4 * P + Nz * Nz; }
        const CT<R> *u = su + cp * Nz;
        for (int zp = 0; zp < Nz; zp++) {
            CT<R> g;
            if (kind == 0) g = (z <= zp) ? blk[z + zp * (zp + 1) / 2] : blk[zp + z * (z + 1) / 2];
            else if (kind == 1) g = blk[asw(z, zp, Nz, AW)];
            else g = blk[asw(zp, z, Nz, AW)];
#pragma unroll
            for (int p = 0; p < 4; p++) cfma(part[p], g, u[p * Z3 + zp]);
        }
        // signs
#pragma unroll
        for (int p = 0; p < 4; p++) {
            const R sxs = (p & 2) ? R(-1) : R(1), ms = (p & 1) ? R(-1) : R(1);
            R sg_ = R(1);
            if ((c == 0 && cp == 1) || (c == 1 && cp == 0)) sg_ = sxs * ms;
            else if (c == 0 && cp == 2) sg_ = sxs;
            else if (c == 2 && cp == 0) sg_ = -sxs;
            else if (c == 1 && cp == 2) sg_ = ms;
            else if (c == 2 && cp == 1) sg_ = -ms;
            acc[p].x += sg_ * part[p].x;
            acc[p].y += sg_ * part[p].y;
        }
    }
    if (q == 0) { acc[2] = czero<CT<R>>(); acc[3] = czero<CT<R>>(); }
    if (r == 0) { acc[1] = czero<CT<R>>(); acc[3] = czero<CT<R>>(); }
#pragma unroll
    for (int p = 0; p < 4; p++) Uhat[unit * 4 * Z3 + p * Z3 + t] = acc[p];
}

// per-cell coefficients (apply_ie_operator_module.F90:66-68, :134):
//   asiga = 2*sqrt(Re sb)/(csiga + conj(sb)),  gsig = (csiga - sb)*asiga
__global__ void k_sigma(const double2 *__restrict__ csiga, const double2 *__restrict__ csigb,
                        const double *__restrict__ sq, double2 *gsig64, double2 *asig64, float2 *gsig32,
                        float2 *asig32, size_t plane, int Nz)
{
    const size_t n = plane * Nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(i / plane);
        const double2 sa = csiga[i], sb = csigb[z];
        const double2 a = cdiv(make_double2(2.0 * sq[z], 0.0), make_double2(sa.x + sb.x, sa.y - sb.y));
        const double2 g = cmul(make_double2(sa.x - sb.x, sa.y - sb.y), a);
        gsig64[i] = g;
        asig64[i] = a;
        gsig32[i] = make_float2((float)g.x, (float)g.y);
        asig32[i] = make_float2((float)a.x, (float)a.y);
    }
}

template <typename R> struct Bufs;
template <> struct Bufs<double> {
    static const double2 *G(IeOp *o) { return o->d_tensor64; }
    static const double2 *gsig(IeOp *o) { return o->d_gsig64; }
    static const double2 *asig(IeOp *o) { return o->d_asig64; }
    static const double *post(IeOp *o) { return o->d_post64; }
    static const double2 *twx(IeOp *o) { return o->d_twx64; }
    static const double2 *twy(IeOp *o) { return o->d_twy64; }
};
template <> struct Bufs<float> {
    static const float2 *G(IeOp *o) { return o->d_tensor32; }
    static const float2 *gsig(IeOp *o) { return o->d_gsig32; }
    static const float2 *asig(IeOp *o) { return o->d_asig32; }
    static const float *post(IeOp *o) { return o->d_post32; }
    static const float2 *twx(IeOp *o) { return o->d_twx32; }
    static const float2 *twy(IeOp *o) { return o->d_twy32; }
};

}  // namespace

static bool uses_ypipe(const IeOp *op, int form)
{
    return op->use_fast_contract && op->ypipe_mode[form] >= 0 && ie_ypipe_supported(op->Nx, op->Ny, op->Nz);
}

int ie_kernel_launch_count_apply(const IeOp *op, int form) { return uses_ypipe(op, form) ? 3 : 5; }

// elements of the spectrum of one vector, and the pipelined pass's counters after it (in 8-byte units, so
// the same count covers them behind a complex64 or a complex128 spectrum)
static size_t spectrum_elems(const IeOp *op) { return (size_t)op->Nx * op->Ny * 4 * 3 * op->Nz; }
static size_t ystate_elems(const IeOp *op) { return (ie_ypipe_state_bytes(op->Nx) + 7) / 8; }

// lines per CTA: tile of at most ~100 KB of shared memory, power of two, <= 32
static int lines_for(int L, size_t es, int cap)
{
    int n = cap >= 1 && cap <= 32 ? cap : 32;
    while (n > 1 && (size_t)(n * (L + 1) + L) * es > 100 * 1024) n >>= 1;
    return n;
}
// threads: one per work item of the larger four-step pass, whole warps, at most 256
static int threads_for(int L, int NL)
{
    int n1 = 2, n2 = 2;
    switch (L) {
    case 4: n1 = 2; n2 = 2; break;
    case 8: n1 = 4; n2 = 2; break;
    case 16: n1 = 4; n2 = 4; break;
    case 32: n1 = 8; n2 = 4; break;
    case 64: n1 = 8; n2 = 8; break;
    case 128: n1 = 16; n2 = 8; break;
    case 256: n1 = 16; n2 = 16; break;
    case 512: n1 = 32; n2 = 16; break;
    default: n1 = 32; n2 = 32; break;
    }
    int t = NL * (n1 > n2 ? n1 : n2);
    t = ((t + 31) / 32) * 32;
    return t > kThreads ? kThreads : t;
}
template <typename K> static void big_smem(K k)
{
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
}

// the register-capped pass kernels apply when the block fits their bounds (PassLB)
template <typename R, int L> static bool use_cap(int nt) { return L <= 256 && nt <= PassLB<R, 1>::T; }

template <typename R, int L, int CAP>
static void launch_x_k(bool fwd, IeOp *op, const VecSet<CT<R>> &vs, CT<R> *U1, cudaStream_t st, const int *gate,
                       dim3 grid, int nt, size_t sm, int NL)
{
    const int Nx = op->Nx, Ny = op->Ny, Nz = op->Nz;
    static bool attr = false;
    if (!attr) { big_smem(k_fx<R, L, CAP>); big_smem(k_bx<R, L, CAP>); attr = true; }
    if (fwd)
        k_fx<R, L, CAP><<<grid, nt, sm, st>>>(vs, Bufs<R>::gsig(op), U1, Bufs<R>::twx(op), Nx, Ny, Nz, NL, gate);
    else
        k_bx<R, L, CAP><<<grid, nt, sm, st>>>(U1, vs, Bufs<R>::asig(op), Bufs<R>::post(op), Bufs<R>::twx(op), Nx,
                                              Ny, Nz, NL, gate);
}

template <typename R, int L>
static void launch_x(bool fwd, IeOp *op, const VecSet<CT<R>> &vs, CT<R> *U1, cudaStream_t st, const int *gate)
{
    const int Nz = op->Nz, ZL = vs.nv * 3 * Nz;
    const size_t es = sizeof(CT<R>);
    const int NL = lines_for(L, es, op->fft_lines[es == sizeof(double2) ? 0 : 1]), nt = threads_for(L, NL);
    const size_t sm = (size_t)(NL * (L + 1) + L) * es;
    dim3 grid((ZL + NL - 1) / NL, op->Ny);
    if (use_cap<R, L>(nt)) launch_x_k<R, L, 1>(fwd, op, vs, U1, st, gate, grid, nt, sm, NL);
    else launch_x_k<R, L, 0>(fwd, op, vs, U1, st, gate, grid, nt, sm, NL);
}

template <typename R, int L, int CAP>
static void launch_y_k(bool fwd, IeOp *op, int nv, CT<R> *U1, CT<R> *Uh, cudaStream_t st, const int *gate,
                       dim3 grid, int nt, size_t sm, int NL)
{
    const int Nx = op->Nx, Ny = op->Ny, Nz = op->Nz;
    static bool attr = false;
    if (!attr) { big_smem(k_fy<R, L, CAP>); big_smem(k_by<R, L, CAP>); attr = true; }
    if (fwd) k_fy<R, L, CAP><<<grid, nt, sm, st>>>(U1, Uh, Bufs<R>::twy(op), Nx, Ny, Nz, NL, nv, gate);
    else k_by<R, L, CAP><<<grid, nt, sm, st>>>(Uh, U1, Bufs<R>::twy(op), Nx, Ny, Nz, NL, nv, gate);
}

template <typename R, int L>
static void launch_y(bool fwd, IeOp *op, int nv, CT<R> *U1, CT<R> *Uh, cudaStream_t st, const int *gate)
{
    const int Nz = op->Nz, ZL = nv * 3 * Nz;
    const size_t es = sizeof(CT<R>);
    const int NL = lines_for(L, es, op->fft_lines[es == sizeof(double2) ? 0 : 1]), nt = threads_for(L, NL);
    const size_t sm = (size_t)(NL * (L + 1) + L) * es;
    dim3 grid((ZL + NL - 1) / NL, 2 * op->Nx);
    if (use_cap<R, L>(nt)) launch_y_k<R, L, 1>(fwd, op, nv, U1, Uh, st, gate, grid, nt, sm, NL);
    else launch_y_k<R, L, 0>(fwd, op, nv, U1, Uh, st, gate, grid, nt, sm, NL);
}

template <typename R>
static void dispatch_x(bool fwd, IeOp *op, const VecSet<CT<R>> &vs, CT<R> *U1, cudaStream_t st, const int *gate)
{
    switch (2 * op->Nx) {
    case 4: launch_x<R, 4>(fwd, op, vs, U1, st, gate); break;
    case 8: launch_x<R, 8>(fwd, op, vs, U1, st, gate); break;
    case 16: launch_x<R, 16>(fwd, op, vs, U1, st, gate); break;
    case 32: launch_x<R, 32>(fwd, op, vs, U1, st, gate); break;
    case 64: launch_x<R, 64>(fwd, op, vs, U1, st, gate); break;
    case 128: launch_x<R, 128>(fwd, op, vs, U1, st, gate); break;
    case 256: launch_x<R, 256>(fwd, op, vs, U1, st, gate); break;
    case 512: launch_x<R, 512>(fwd, op, vs, U1, st, gate); break;
    case 1024: launch_x<R, 1024>(fwd, op, vs, U1, st, gate); break;
    }
}
template <typename R>
static void dispatch_y(bool fwd, IeOp *op, int nv, CT<R> *U1, CT<R> *Uh, cudaStream_t st, const int *gate)
{
    switch (2 * op->Ny) {
    case 4: launch_y<R, 4>(fwd, op, nv, U1, Uh, st, gate); break;
    case 8: launch_y<R, 8>(fwd, op, nv, U1, Uh, st, gate); break;
    case 16: launch_y<R, 16>(fwd, op, nv, U1, Uh, st, gate); break;
    case 32: launch_y<R, 32>(fwd, op, nv, U1, Uh, st, gate); break;
    case 64: launch_y<R, 64>(fwd, op, nv, U1, Uh, st, gate); break;
    case 128: launch_y<R, 128>(fwd, op, nv, U1, Uh, st, gate); break;
    case 256: launch_y<R, 256>(fwd, op, nv, U1, Uh, st, gate); break;
    case 512: launch_y<R, 512>(fwd, op, nv, U1, Uh, st, gate); break;
    case 1024: launch_y<R, 1024>(fwd, op, nv, U1, Uh, st, gate); break;
    }
}

// The five kernels over the scratch pair (U1, Uh); every element of both is written before it is
// read, so neither has to start at zero.
template <typename R>
static int ie_apply_core(IeOp *op, const CT<R> *d_in, CT<R> *d_out, cudaStream_t st, const int *gate, CT<R> *U1,
                         CT<R> *Uh)
{
    const int Nx = op->Nx, Ny = op->Ny, Nz = op->Nz, Z3 = 3 * Nz;
    const size_t es = sizeof(CT<R>);
    const CT<R> *G = Bufs<R>::G(op);
    if (!G || !U1 || !Uh) return G2_ERR_STATE;
    VecSet<CT<R>> vs{{d_in, nullptr}, {d_out, nullptr}, 1};
    const int form = sizeof(R) == 8 ? 0 : 1;
    // contraction (bracketed by events when kernel timing is on; never inside a stream capture)
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    const bool timed = op->time_contract && op->evc0 &&
                       cudaStreamIsCapturing(st, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone;
    dispatch_x<R>(true, op, vs, U1, st, gate);
    if (uses_ypipe(op, form)) {
        // y-FFT, contraction and inverse y-FFT in one pass, the spectrum as L2-resident scratch
        int *state = reinterpret_cast<int *>(Uh + spectrum_elems(op));
        if (timed) cudaEventRecord(op->evc0, st);
        const int rc = ie_ypipe(op, form, G, U1, Uh, state, st, gate);
        if (rc) return rc;
        if (timed) cudaEventRecord(op->evc1, st);
        dispatch_x<R>(false, op, vs, U1, st, gate);
        g2_count_launches(3);
        G2_CUDA_CHECK(cudaGetLastError());
        return G2_OK;
    }
    dispatch_y<R>(true, op, 1, U1, Uh, st, gate);
    if (timed) cudaEventRecord(op->evc0, st);
    int rc_fast = G2_ERR_UNSUPPORTED;
    if (op->use_fast_contract) {
        if (sizeof(R) == 8)
            rc_fast = ie_contract_fast64(reinterpret_cast<const double2 *>(G), reinterpret_cast<double2 *>(Uh), Nx, Ny,
                                         Nz, op->d_err, st, op->contract_variant[0], gate);
        else
            rc_fast = ie_contract_fast32(reinterpret_cast<const float2 *>(G), reinterpret_cast<float2 *>(Uh), Nx, Ny,
                                         Nz, op->d_err, st, op->contract_variant[1], gate);
        if (rc_fast != G2_OK && rc_fast != G2_ERR_UNSUPPORTED) return rc_fast;
    }
    if (rc_fast != G2_OK) {
        const int T = op->Tunit();
        const size_t sm = ((size_t)T + 4 * Z3) * es;
        const int threads = ((Z3 + 31) / 32) * 32;
        k_contract<R><<<(unsigned)op->units(), threads, sm, st>>>(G, Uh, Nx, Ny, Nz, gate);
    }
    if (timed) cudaEventRecord(op->evc1, st);
    dispatch_y<R>(false, op, 1, U1, Uh, st, gate);
    dispatch_x<R>(false, op, vs, U1, st, gate);
    g2_count_launches(5);
    G2_CUDA_CHECK(cudaGetLastError());
    return G2_OK;
}

template <typename R>
static int ie_apply_device(IeOp *op, const CT<R> *d_in, CT<R> *d_out, cudaStream_t st, const int *gate)
{
    return ie_apply_core<R>(op, d_in, d_out, st, gate, reinterpret_cast<CT<R> *>(op->scratch.U1),
                            reinterpret_cast<CT<R> *>(op->scratch.Uhat));
}

int ie_apply_device64(IeOp *op, const double2 *d_in, double2 *d_out, cudaStream_t st, const int *gate)
{
    return ie_apply_device<double>(op, d_in, d_out, st, gate);
}
namespace {
__global__ void k_c128_to_c64(const double2 *__restrict__ a, float2 *__restrict__ b, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = make_float2((float)a[i].x, (float)a[i].y);
}
__global__ void k_c64_to_c128(const float2 *__restrict__ a, double2 *__restrict__ b, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = make_double2((double)a[i].x, (double)a[i].y);
}
}  // namespace

// The reference-facing apply in the operator's precision mode 1: complex128 in and out, complex64 inside.
int ie_apply_host_mixed(IeOp *op, const double2 *d_in, double2 *d_out, cudaStream_t st)
{
    const long long n = (long long)op->nvec();
    if (!op->d_vin32) {
        G2_CUDA_CHECK(cudaMalloc(&op->d_vin32, n * sizeof(float2)));
        G2_CUDA_CHECK(cudaMalloc(&op->d_vout32, n * sizeof(float2)));
    }
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_c128_to_c64<<<blocks, 256, 0, st>>>(d_in, op->d_vin32, n);
    G2_CUDA_CHECK(cudaGetLastError());
    int rc = ie_apply_device32(op, op->d_vin32, op->d_vout32, st);
    if (rc) return rc;
    k_c64_to_c128<<<blocks, 256, 0, st>>>(op->d_vout32, d_out, n);
    G2_CUDA_CHECK(cudaGetLastError());
    g2_count_launches(2);
    return G2_OK;
}

int ie_apply_device32(IeOp *op, const float2 *d_in, float2 *d_out, cudaStream_t st, const int *gate)
{
    return ie_apply_device<float>(op, d_in, d_out, st, gate);
}

size_t ie_apply_scratch_elems(const IeOp *op, size_t *n_u1)
{
    const size_t u1 = (size_t)2 * op->Nx * 3 * op->Nz * op->Ny;
    if (n_u1) *n_u1 = u1;
    return u1 + spectrum_elems(op) + ystate_elems(op);
}
int ie_apply_device64_scratch(IeOp *op, const double2 *d_in, double2 *d_out, cudaStream_t st, double2 *U1,
                              double2 *Uhat)
{
    return ie_apply_core<double>(op, d_in, d_out, st, nullptr, U1, Uhat);
}
int ie_apply_device32_scratch(IeOp *op, const float2 *d_in, float2 *d_out, cudaStream_t st, float2 *U1,
                              float2 *Uhat)
{
    return ie_apply_core<float>(op, d_in, d_out, st, nullptr, U1, Uhat);
}

static int set_smem_attrs(IeOp *op)
{
    static bool done = false;
    if (done) return G2_OK;
    const int big = 227 * 1024;
    G2_CUDA_CHECK(cudaFuncSetAttribute(k_contract<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    G2_CUDA_CHECK(cudaFuncSetAttribute(k_contract<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    (void)op;
    done = true;
    return G2_OK;
}

int ie_alloc_scratch(IeOp *op)
{
    const size_t n_u1 = (size_t)2 * op->Nx * 3 * op->Nz * op->Ny;
    const size_t n_uh = spectrum_elems(op) + ystate_elems(op);
    if (!op->scratch.U1) G2_CUDA_CHECK(cudaMalloc(&op->scratch.U1, n_u1 * sizeof(double2)));
    if (!op->scratch.Uhat) G2_CUDA_CHECK(cudaMalloc(&op->scratch.Uhat, n_uh * sizeof(double2)));
    return set_smem_attrs(op);
}

// twiddles exp(-2 pi i j / L), j < L, rounded from long double
static int make_tw(int L, double2 **d64, float2 **d32)
{
    std::vector<double2> h64(L);
    std::vector<float2> h32(L);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int j = 0; j < L; j++) {
        long double a = -2.0L * pi * (long double)j / (long double)L;
        h64[j] = make_double2((double)cosl(a), (double)sinl(a));
        h32[j] = make_float2((float)cosl(a), (float)sinl(a));
    }
    G2_CUDA_CHECK(cudaMalloc(d64, sizeof(double2) * L));
    G2_CUDA_CHECK(cudaMalloc(d32, sizeof(float2) * L));
    G2_CUDA_CHECK(cudaMemcpy(*d64, h64.data(), sizeof(double2) * L, cudaMemcpyHostToDevice));
    G2_CUDA_CHECK(cudaMemcpy(*d32, h32.data(), sizeof(float2) * L, cudaMemcpyHostToDevice));
    // a pageable cudaMemcpy may return before its DMA lands, and the operator's non-blocking stream is
    // not ordered after the legacy stream: wait for it here
    G2_CUDA_CHECK(cudaStreamSynchronize(cudaStreamLegacy));
    return G2_OK;
}

int ie_make_twiddles(IeOp *op)
{
    int rc = make_tw(2 * op->Nx, &op->d_twx64, &op->d_twx32);
    if (rc) return rc;
    return make_tw(2 * op->Ny, &op->d_twy64, &op->d_twy32);
}

int ie_prepare_sigma(IeOp *op, cudaStream_t st)
{
    const int Nz = op->Nz;
    const size_t n = op->cells();
    if (!op->d_gsig64) {
        G2_CUDA_CHECK(cudaMalloc(&op->d_gsig64, n * sizeof(double2)));
        G2_CUDA_CHECK(cudaMalloc(&op->d_asig64, n * sizeof(double2)));
        G2_CUDA_CHECK(cudaMalloc(&op->d_gsig32, n * sizeof(float2)));
        G2_CUDA_CHECK(cudaMalloc(&op->d_asig32, n * sizeof(float2)));
        G2_CUDA_CHECK(cudaMalloc(&op->d_post64, 2 * Nz * sizeof(double)));
        G2_CUDA_CHECK(cudaMalloc(&op->d_post32, 2 * Nz * sizeof(float)));
    }
    std::vector<double> post(2 * Nz);
    std::vector<float> post32(2 * Nz);
    const double N = 4.0 * op->Nx * op->Ny;
    for (int z = 0; z < Nz; z++) {
        post[z] = op->sqsigb[z];
        post[Nz + z] = 1.0 / (op->dz[z] * N);
        post32[z] = (float)post[z];
        post32[Nz + z] = (float)post[Nz + z];
    }
    G2_CUDA_CHECK(cudaMemcpyAsync(op->d_post64, post.data(), 2 * Nz * sizeof(double), cudaMemcpyHostToDevice, st));
    G2_CUDA_CHECK(cudaMemcpyAsync(op->d_post32, post32.data(), 2 * Nz * sizeof(float), cudaMemcpyHostToDevice, st));
    double2 *d_csigb = nullptr;
    double *d_sq = nullptr;
    G2_CUDA_CHECK(cudaMalloc(&d_csigb, Nz * sizeof(double2)));
    G2_CUDA_CHECK(cudaMalloc(&d_sq, Nz * sizeof(double)));
    G2_CUDA_CHECK(cudaMemcpyAsync(d_csigb, op->csigb.data(), Nz * sizeof(double2), cudaMemcpyHostToDevice, st));
    G2_CUDA_CHECK(cudaMemcpyAsync(d_sq, op->sqsigb.data(), Nz * sizeof(double), cudaMemcpyHostToDevice, st));
    k_sigma<<<592, 256, 0, st>>>(op->d_csiga, d_csigb, d_sq, op->d_gsig64, op->d_asig64, op->d_gsig32, op->d_asig32,
                                 (size_t)op->Nx * op->Ny, Nz);
    G2_CUDA_CHECK(cudaGetLastError());
    G2_CUDA_CHECK(cudaStreamSynchronize(st));
    cudaFree(d_csigb);
    cudaFree(d_sq);
    return G2_OK;
}

size_t ie_pair_scratch_elems(const IeOp *op, size_t *n_u1)
{
    size_t u1 = 0;
    const size_t all = ie_apply_scratch_elems(op, &u1);
    if (n_u1) *n_u1 = 2 * u1;
    return 2 * all;
}
// Two complex64 vectors of one operator in one apply: the FFT passes run over both vectors' lines and the
// contraction applies each tensor unit, read once, to both spectra.  Returns G2_ERR_UNSUPPORTED (nothing
// launched) when no paired contraction exists for the grid.
int ie_apply_pair32(IeOp *op, const float2 *in0, const float2 *in1, float2 *out0, float2 *out1, cudaStream_t st,
                    float2 *U1, float2 *Uh)
{
    if (!op->use_fast_contract || !ie_contract_pair32_supported(op->Nx, op->Ny, op->Nz)) return G2_ERR_UNSUPPORTED;
    if (!op->d_tensor32 || !U1 || !Uh) return G2_ERR_STATE;
    VecSet<float2> vs{{in0, in1}, {out0, out1}, 2};
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    const bool timed = op->time_contract && op->evc0 &&
                       cudaStreamIsCapturing(st, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone;
    dispatch_x<float>(true, op, vs, U1, st, nullptr);
    if (uses_ypipe(op, 2)) {
        int *state = reinterpret_cast<int *>(Uh + 2 * spectrum_elems(op));
        if (timed) cudaEventRecord(op->evc0, st);
        const int rc = ie_ypipe(op, 2, op->d_tensor32, U1, Uh, state, st, nullptr);
        if (rc) return rc;
        if (timed) cudaEventRecord(op->evc1, st);
        dispatch_x<float>(false, op, vs, U1, st, nullptr);
        g2_count_launches(3);
        G2_CUDA_CHECK(cudaGetLastError());
        return G2_OK;
    }
    dispatch_y<float>(true, op, 2, U1, Uh, st, nullptr);
    if (timed) cudaEventRecord(op->evc0, st);
    const int rc = ie_contract_pair32(op->d_tensor32, Uh, op->Nx, op->Ny, op->Nz, op->d_err, st, nullptr,
                                      op->contract_variant[2]);
    if (rc) return rc;
    if (timed) cudaEventRecord(op->evc1, st);
    dispatch_y<float>(false, op, 2, U1, Uh, st, nullptr);
    dispatch_x<float>(false, op, vs, U1, st, nullptr);
    g2_count_launches(5);
    G2_CUDA_CHECK(cudaGetLastError());
    return G2_OK;
}
int ie_pair_scratch(IeOp *op, float2 **U1, float2 **Uh)
{
    size_t n_u1 = 0;
    const size_t n_all = ie_pair_scratch_elems(op, &n_u1);
    if (!op->pair_scratch.U1) G2_CUDA_CHECK(cudaMalloc(&op->pair_scratch.U1, n_u1 * sizeof(float2)));
    if (!op->pair_scratch.Uhat) G2_CUDA_CHECK(cudaMalloc(&op->pair_scratch.Uhat, (n_all - n_u1) * sizeof(float2)));
    *U1 = reinterpret_cast<float2 *>(op->pair_scratch.U1);
    *Uh = reinterpret_cast<float2 *>(op->pair_scratch.Uhat);
    return G2_OK;
}
