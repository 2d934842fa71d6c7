// Pieces of the barrier-free Green's-tensor contraction shared by its kernels (contract.cu: the
// stand-alone k_contract_wl; ypipe.cu: the form fused with the y-transforms).
//
// wl_unit_sums: one lane's partial sums over its j-slice for one (kx-pair, ky-pair) unit.  Lane (z, s)
// owns row z and sums j = s, s + SL, s + 2 SL, ... of the six Green's blocks (xx, xy, yy, zz packed upper,
// xz, yz full and XOR-swizzled) applied to the PTS = 4 NP spectral points of the unit with the reference's
// sign table (apply_ie_operator_module.F90:278-291).  The tensor unit gb and the points ub ([pt][c][j],
// pt = slot * NP + vector) sit in shared memory.
// wl_unit_store: the recursive-halving reduction of the SL slices of a row across the warp's lanes, and
// the store of each lane's share of the outputs, with the Nyquist points (q = 0 slot bit 2, r = 0 slot
// bit 1) zeroed as in the reference.
#pragma once
#include "common.cuh"
#include "tma.cuh"

// (a.x*b.x + c.x, a.y*b.y + c.y) in one packed FP32 instruction
G2_D float2 ffma2(float2 a, float2 b, float2 c)
{
    union U { float2 f; unsigned long long u; } ua, ub, uc, ud;
    ua.f = a;
    ub.f = b;
    uc.f = c;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(ud.u) : "l"(ua.u), "l"(ub.u), "l"(uc.u));
    return ud.f;
}

template <typename R> struct V2;
template <> struct V2<double> { using T = double2; };
template <> struct V2<float> { using T = float2; };

template <int NZ>
G2_D int sym_idx(int i, int j) { return i <= j ? i + j * (j + 1) / 2 : j + i * (i + 1) / 2; }

// one halving step over lane bit B of the slice index, then the next; v[0, LEN) is still held
template <int B, int LEN, int ZW, int SL, int NR, typename R>
G2_D void halve_slices(R (&v)[NR], int s, int &f0)
{
    if constexpr ((1 << B) < SL) {
        constexpr int HALF = LEN / 2;
        const bool up = (s >> B) & 1;
#pragma unroll
        for (int i = 0; i < HALF; i++) {
            const R send = up ? v[i] : v[HALF + i];
            const R keep = up ? v[HALF + i] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, ZW << B);
        }
        if (up) f0 += HALF;
        halve_slices<B + 1, HALF, ZW, SL, NR>(v, s, f0);
    }
}

// Spin (bounded, 2 s) until ticket it-1 has been passed; on timeout records `code` in *err.
G2_D bool wait_ticket(const int *passed, int it, int *err, int code = 17)
{
    const volatile int *p = passed;
    if (*p >= it) return true;
    const uint64_t t0 = globaltimer_ns();
    while (*p < it) {
        if (globaltimer_ns() - t0 > 2000000000ull) {
            atomicCAS(err, 0, code);
            return false;
        }
    }
    return true;
}

// VS: the NP vectors split over VS lane groups (1: every lane holds all 4 NP points; NP: one vector per lane,
// 4 points).  A lane of vector group vv holds the points (slot, vector vv * NP / VS + i); fewer points per lane
// means fewer live accumulators and more resident warps, at the price of the tensor elements being read by
// VS lanes instead of one.
template <int NP, int VS> struct LanePts {
    static_assert(NP % VS == 0, "the vector split must divide the vectors");
    static constexpr int NPL = NP / VS;   // vectors per lane
    static constexpr int PL = 4 * NPL;    // points per lane
    // global point (slot * NP + vector) of the lane's local point p
    static G2_HD int gp(int p, int vv) { return (p / NPL) * NP + vv * NPL + p % NPL; }
};

// UR: j iterations unrolled together (4 let the paired complex64 tile overlap more shared-memory loads with its
// FMAs: 192.6 against 199.3 us at 128x128x32, at 167 instead of 157 registers)
template <typename R, int NZ, int SL, int NP, bool M4, bool PK, int VS = 1, int UR = 2>
G2_D void wl_unit_sums(const typename V2<R>::T *__restrict__ gb, const typename V2<R>::T *__restrict__ ub, int z,
                       int s, R (&v)[2 * 3 * LanePts<NP, VS>::PL], int vv = 0)
{
    using C2 = typename V2<R>::T;
    using LP = LanePts<NP, VS>;
    constexpr int PTS = LP::PL, P = NZ * (NZ + 1) / 2, JS = NZ / SL;
    constexpr int AW = sizeof(R) == 8 ? asw_width64(NZ) : asw_width32(NZ);
    static_assert(!PK || (sizeof(R) == 4 && !M4), "packed pairs are a complex64 3-multiply form");
    constexpr int NA = M4 ? 2 : 3;
    R acc[3][PTS][NA];
    C2 accp[3][PTS];  // PK: (t1, t2) of the 3-multiply form
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int p = 0; p < PTS; p++) {
            accp[c][p] = C2{R(0), R(0)};
#pragma unroll
            for (int k = 0; k < NA; k++) acc[c][p][k] = R(0);
        }
    const C2 *gxx = gb, *gxy = gb + P, *gyy = gb + 2 * P, *gzz = gb + 3 * P;
    const C2 *gxz = gb + 4 * P, *gyz = gb + 4 * P + NZ * NZ;
#pragma unroll UR
    for (int jj = 0; jj < JS; jj++) {
        const int j = jj * SL + s;
        const int si = sym_idx<NZ>(z, j);
        const int a_zj = asw(z, j, NZ, AW), a_jz = asw(j, z, NZ, AW);
        const C2 e[8] = {gxx[si], gxy[si], gyy[si], gzz[si], gxz[a_zj], gyz[a_zj], gxz[a_jz], gyz[a_jz]};
        C2 en[8];  // PK: negated copies (only the ones a negative sign uses survive compilation)
#pragma unroll
        for (int k = 0; k < 8; k++) en[k] = C2{-e[k].x, -e[k].y};
        C2 u[PTS][3];
        R ue[PTS][3];
#pragma unroll
        for (int p = 0; p < PTS; p++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                u[p][c] = ub[(LP::gp(p, vv) * 3 + c) * NZ + j];
                ue[p][c] = u[p][c].x + u[p][c].y;
            }
        // sign table as in k_contract_tma; point p = slot * NP + vector, slot bits (sx, m)
#define G2_TERM_L(C, K, IN, SGN)                                                 \
{                                                                            \
    const R es_ = e[K].x + e[K].y;                                           \
    _Pragma("unroll") for (int p = 0; p < PTS; p++)                          \
    {                                                                        \
        const int sl_ = p / LP::NPL;                                         \
        const R sx = (sl_ & 2) ? R(-1) : R(1);                               \
        const R m = (sl_ & 1) ? R(-1) : R(1);                                \
        const R sg = (SGN);                                                  \
        if constexpr (PK) {                                                  \
            accp[C][p] = ffma2(sg < R(0) ? en[K] : e[K], u[p][IN], accp[C][p]); \
            acc[C][p][NA - 1] = fma(sg * es_, ue[p][IN], acc[C][p][NA - 1]); \
        } else if constexpr (M4) {                                           \
            acc[C][p][0] = fma(sg * e[K].x, u[p][IN].x, acc[C][p][0]);       \
            acc[C][p][0] = fma(-sg * e[K].y, u[p][IN].y, acc[C][p][0]);      \
            acc[C][p][1] = fma(sg * e[K].x, u[p][IN].y, acc[C][p][1]);       \
            acc[C][p][1] = fma(sg * e[K].y, u[p][IN].x, acc[C][p][1]);       \
        } else {                                                             \
            acc[C][p][0] = fma(sg * e[K].x, u[p][IN].x, acc[C][p][0]);       \
            acc[C][p][1] = fma(sg * e[K].y, u[p][IN].y, acc[C][p][1]);       \
            acc[C][p][NA - 1] = fma(sg * es_, ue[p][IN], acc[C][p][NA - 1]); \
        }                                                                    \
    }                                                                        \
}
        G2_TERM_L(0, 0, 0, R(1))
        G2_TERM_L(1, 1, 0, sx * m)
        G2_TERM_L(2, 6, 0, -sx)
        G2_TERM_L(0, 1, 1, sx * m)
        G2_TERM_L(1, 2, 1, R(1))
        G2_TERM_L(2, 7, 1, -m)
        G2_TERM_L(0, 4, 2, sx)
        G2_TERM_L(1, 5, 2, m)
        G2_TERM_L(2, 3, 2, R(1))
#undef G2_TERM_L
    }
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int p = 0; p < PTS; p++) {
            if constexpr (PK) {
                const R t1 = accp[c][p].x, t2 = accp[c][p].y, t3 = acc[c][p][NA - 1];
                v[2 * (c * PTS + p)] = t1 - t2;
                v[2 * (c * PTS + p) + 1] = t3 - t1 - t2;
            } else if constexpr (M4) {
                v[2 * (c * PTS + p)] = acc[c][p][0];
                v[2 * (c * PTS + p) + 1] = acc[c][p][1];
            } else {
                const R t1 = acc[c][p][0], t2 = acc[c][p][1], t3 = acc[c][p][NA - 1];
                v[2 * (c * PTS + p)] = t1 - t2;
                v[2 * (c * PTS + p) + 1] = t3 - t1 - t2;
            }
        }
}

// lanes: zl + ZW * (s + SL * vv), ZW = 32 / (SL * VS) rows per warp
template <typename R, int NZ, int SL, int NP, int VS = 1>
G2_D void wl_unit_store(R (&v)[2 * 3 * LanePts<NP, VS>::PL], int s, int q, int r, typename V2<R>::T *dst, int vv = 0)
{
    using C2 = typename V2<R>::T;
    using LP = LanePts<NP, VS>;
    constexpr int PTS = LP::PL, NR = 2 * 3 * PTS, HR = NR / SL, ZW = 32 / (SL * VS);
    int f0 = 0;  // first flat output index this lane keeps
    halve_slices<0, NR, ZW, SL, NR>(v, s, f0);
#pragma unroll
    for (int i = 0; i < HR; i += 2) {
        const int k = (f0 + i) >> 1, c = k / PTS, p = k - c * PTS, sl = p / LP::NPL;
        C2 o{v[i], v[i + 1]};
        if ((q == 0 && (sl & 2)) || (r == 0 && (sl & 1))) o = C2{R(0), R(0)};
        dst[(LP::gp(p, vv) * 3 + c) * NZ] = o;
    }
}
