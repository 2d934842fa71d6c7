// Green's-tensor contraction at every (kx-pair, ky-pair) unit: the hot loop of the apply.
//
// Restates VERTICAL_MULT_GENERAL / _ZERO (apply_ie_operator_module.F90:265-374): at each unit (q,r)
// the six Nz x Nz blocks (xx, xy, yy, zz symmetric packed; xz, yz full) multiply the 3-component
// spectrum at the four points (+-kx, +-ky) with the reference's sign table.  One tensor read serves
// the four points (the reference does the same with its slot pair and MirrorY = +-1).
//
// Design (persistent, one CTA per SM):
//   * producer warp: one lane streams B units of tensor + their 4-point spectra per stage into shared
//     memory with cp.async.bulk (TMA engine), tensor with an L2 evict_first hint so that it does not
//     push the spectra and the Krylov vectors out of L2 (the spectra get no hint: pinning them with
//     evict_last cost the solver's vector kernels their L2 hits); NSTAGE-deep mbarrier ring;
//   * consumer warps: thread (b, s, z) owns row z of unit b for all 3 components and 4 points and sums
//     over the j-slice s; complex products use 3 real multiplies (T1=a c, T2=b d, T3=(a+b)(c+d);
//     re=T1-T2, im=T3-T1-T2), 25% fewer FMAs than 4-multiply complex arithmetic, which matters because
//     the FP64 contraction sits at the B200 FP64 ridge; FMAs are issued term-major so consecutive ones
//     update independent accumulators; the 4-point inputs are broadcast reads of the staged spectrum;
//     slice partials are reduced through the drained stage buffer; Nyquist points are zeroed as in
//     the reference.
// Every mbarrier wait is bounded (2 s); on timeout the kernel records an error code and returns after
// the producer has waited (bounded) for its copies in flight.
#include "common.cuh"
#include "ie_internal.h"
#include "tma.cuh"
#include "contract_wl.cuh"

namespace {

template <typename R, int NZ, int S, int B, int NSTAGE, int NP = 1, bool SPLIT = false, int MINB = 1>
struct CfgT {
    static constexpr int P = NZ * (NZ + 1) / 2;
    static constexpr int T = 4 * P + 2 * NZ * NZ;        // complex per unit
    static constexpr int Z3 = 3 * NZ;
    static constexpr int PTS = 4 * NP;                     // spectral points per unit: 4 slots x NP vectors
    static constexpr int VT = SPLIT ? NP : 1;              // vectors spread over threads
    static constexpr int PR = PTS / VT;                    // points held in one thread's registers
    static constexpr int NC = B * S * NZ * VT;             // consumer threads
    static constexpr int NTHREADS = NC + 32;
    static constexpr int JS = NZ / S;                      // j per slice
    static constexpr int ES = 2 * sizeof(R);               // bytes per complex
    static constexpr int TBYTES = B * T * ES;
    static constexpr int UBYTES = B * PTS * Z3 * ES;
    static constexpr int STAGE_BYTES = TBYTES + UBYTES;
    static constexpr int RED_BYTES = S * B * PTS * 3 * NZ * ES;
    static constexpr int SMEM = NSTAGE * STAGE_BYTES + 2 * NSTAGE * 8;
    static_assert(NZ % S == 0, "slices must divide Nz");
    static_assert(NC % 32 == 0, "consumer threads must be whole warps");
    static_assert(RED_BYTES <= TBYTES, "reduction buffer reuses the drained tensor stage");
    static_assert(STAGE_BYTES % 16 == 0 && TBYTES % 16 == 0, "bulk copies need 16-byte multiples");
    static_assert(SMEM <= 232448, "exceeds the 227 KB dynamic shared memory of one CTA");
    static_assert(MINB * (SMEM + 1024) <= 233472, "MINB CTAs do not fit the SM's shared memory");
};

// NP > 1: NP vectors share every tensor unit (several right-hand sides of one operator); the spectrum of
// a unit is [slot][vector][3Nz] and point pt = slot * NP + vector.  SPLIT: each thread computes the 4
// points of one vector (threads (b, v, s, z)); otherwise each thread holds all 4*NP points.
// PK (complex64 only): the 3-multiply form with its first two products as one packed fma.rn.f32x2 per
// term and point, (e.x, e.y) * (u.x, u.y) + (t1, t2), and the third, (e.x + e.y)(u.x + u.y), as a scalar
// FMA: two instructions per complex multiply-add instead of three; a negative sign uses a negated copy
// of the tensor element.
// M4: 4-multiply complex products (two accumulators per output instead of three: 118 registers instead
// of 142, so three FP64 CTAs fit on an SM, for 12 % more FMAs).  At 128x128x32 it gives 0.395 ms per
// FP64 apply against 0.388 ms for the 3-multiply tile with a 3-stage ring: occupancy is not what limits
// the FP64 contraction there, so the tuner keeps the 3-multiply form.
template <typename R, int NZ, int S, int B, int NSTAGE, int NP, bool SPLIT, int MINB, bool M4, bool PK>
__global__ void __launch_bounds__(CfgT<R, NZ, S, B, NSTAGE, NP, SPLIT, MINB>::NTHREADS, MINB)
    k_contract_tma(const typename V2<R>::T *__restrict__ G, typename V2<R>::T *__restrict__ Uhat, int Ny,
                   long long nbatches, int *err, const int *gate)
{
    if (gate && *gate == 0) return;  // uniform across the CTA: nothing has been issued yet
    using Cfg = CfgT<R, NZ, S, B, NSTAGE, NP, SPLIT, MINB>;
    constexpr int PTS = Cfg::PTS, PR = Cfg::PR;
    using C2 = typename V2<R>::T;
    constexpr int AW = sizeof(R) == 8 ? asw_width64(NZ) : asw_width32(NZ);
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *stages = smem;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + NSTAGE * Cfg::STAGE_BYTES);
    uint64_t *empty = full + NSTAGE;

    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], Cfg::NC);
        }
        fence_mbar_init();
    }
    __syncthreads();

    const long long first = blockIdx.x, stride = gridDim.x;
    const long long my_n = first < nbatches ? (nbatches - 1 - first) / stride + 1 : 0;

    if (tid >= Cfg::NC) {
        // ------------------------------- producer warp -------------------------------
        if (tid == Cfg::NC) {
            const uint64_t pol_t = l2_policy_evict_first();
            const uint64_t pol_u = l2_policy_evict_normal();
            long long issued = 0;
            bool ok = true;
            for (long long it = 0; it < my_n; it++) {
                const int slot = (int)(it % NSTAGE);
                const uint32_t round = (uint32_t)(it / NSTAGE);
                if (it >= NSTAGE) {
                    if (!mbar_wait_bounded(&empty[slot], (round - 1) & 1, err, 11)) { ok = false; break; }
                }
                const long long batch = first + it * stride;
                unsigned char *st = stages + slot * Cfg::STAGE_BYTES;
                mbar_arrive_expect_tx(&full[slot], Cfg::STAGE_BYTES);
                bulk_g2s(st, G + batch * (long long)B * Cfg::T, Cfg::TBYTES, &full[slot], pol_t);
                bulk_g2s(st + Cfg::TBYTES, Uhat + batch * (long long)B * PTS * Cfg::Z3, Cfg::UBYTES, &full[slot], pol_u);
                issued++;
            }
            if (!ok) {
                // drain: every issued copy must land before the CTA may exit
                for (long long it = (issued > NSTAGE ? issued - NSTAGE : 0); it < issued; it++)
                    mbar_wait_bounded(&full[it % NSTAGE], (uint32_t)(it / NSTAGE) & 1, err, 12);
            }
        }
        return;
    }

    // ------------------------------- consumers -------------------------------
    const int z = tid % NZ;
    const int s = (tid / NZ) % S;
    const int v = SPLIT ? (tid / (NZ * S)) % NP : 0;
    const int b = tid / (NZ * S * Cfg::VT);
    for (long long it = 0; it < my_n; it++) {
        const int slot = (int)(it % NSTAGE);
        const uint32_t round = (uint32_t)(it / NSTAGE);
        if (!mbar_wait_bounded(&full[slot], round & 1, err, 13)) return;
        const long long batch = first + it * stride;
        unsigned char *st = stages + slot * Cfg::STAGE_BYTES;
        const C2 *gt = reinterpret_cast<const C2 *>(st);
        const C2 *uh = reinterpret_cast<const C2 *>(st + Cfg::TBYTES);
        static_assert(!PK || (sizeof(R) == 4 && !M4), "packed pairs are a complex64 3-multiply form");
        constexpr int NA = M4 ? 2 : 3;
        R acc[3][PR][NA];
        C2 accp[3][PR];  // PK: (t1, t2) of the 3-multiply form
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int p = 0; p < PR; p++) accp[c][p] = C2{R(0), R(0)};
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int p = 0; p < PR; p++)
#pragma unroll
                for (int k = 0; k < NA; k++) acc[c][p][k] = R(0);

        const C2 *gb = gt + b * Cfg::T;
        const C2 *gxx = gb, *gxy = gb + Cfg::P, *gyy = gb + 2 * Cfg::P, *gzz = gb + 3 * Cfg::P;
        const C2 *gxz = gb + 4 * Cfg::P, *gyz = gb + 4 * Cfg::P + NZ * NZ;
        const C2 *ub = uh + b * PTS * Cfg::Z3;  // [pt][c][j], broadcast reads
#pragma unroll 2
        for (int jj = 0; jj < Cfg::JS; jj++) {
            const int j = s * Cfg::JS + jj;
            const int si = sym_idx<NZ>(z, j);
            const int a_zj = asw(z, j, NZ, AW), a_jz = asw(j, z, NZ, AW);
            const C2 e[8] = {gxx[si], gxy[si], gyy[si], gzz[si], gxz[a_zj], gyz[a_zj], gxz[a_jz], gyz[a_jz]};
            C2 en[8];  // PK: negated copies (only the ones a negative sign uses survive compilation)
#pragma unroll
            for (int k = 0; k < 8; k++) en[k] = C2{-e[k].x, -e[k].y};
            C2 u[PR][3];
            R ue[PR][3];
#pragma unroll
            for (int p = 0; p < PR; p++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    u[p][c] = ub[((SPLIT ? p * NP + v : p) * 3 + c) * NZ + j];
                    ue[p][c] = u[p][c].x + u[p][c].y;
                }
            // term-major: each term updates 3*PTS independent accumulators (PTS points x 3 partial products)
#define G2_TERM(C, K, IN, SGN)                                                   \
    {                                                                            \
        const R es_ = e[K].x + e[K].y;                                           \
        _Pragma("unroll") for (int p = 0; p < PR; p++)                           \
        {                                                                        \
            const int sl_ = SPLIT ? p : p / NP;                                  \
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
            // out x: xx Ux + (sx m) xy Uy + sx xz Uz
            // out y: (sx m) xy Ux + yy Uy + m yz Uz
            // out z: -sx xz^T Ux - m yz^T Uy + zz Uz
            G2_TERM(0, 0, 0, R(1))
            G2_TERM(1, 1, 0, sx * m)
            G2_TERM(2, 6, 0, -sx)
            G2_TERM(0, 1, 1, sx * m)
            G2_TERM(1, 2, 1, R(1))
            G2_TERM(2, 7, 1, -m)
            G2_TERM(0, 4, 2, sx)
            G2_TERM(1, 5, 2, m)
            G2_TERM(2, 3, 2, R(1))
#undef G2_TERM
        }
        named_bar_sync(1, Cfg::NC);  // all reads of this stage's tensor and inputs are done
        // slice partials into the drained tensor area: red[s][b][pt][c][z]
        C2 *red = reinterpret_cast<C2 *>(st);
#pragma unroll
        for (int p = 0; p < PR; p++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                C2 o;
                if constexpr (PK) {
                    const R t1 = accp[c][p].x, t2 = accp[c][p].y, t3 = acc[c][p][NA - 1];
                    o.x = t1 - t2;
                    o.y = t3 - t1 - t2;
                } else if constexpr (M4) {
                    o.x = acc[c][p][0];
                    o.y = acc[c][p][1];
                } else {
                    const R t1 = acc[c][p][0], t2 = acc[c][p][1], t3 = acc[c][p][NA - 1];
                    o.x = t1 - t2;
                    o.y = t3 - t1 - t2;
                }
                red[(((s * B + b) * PTS + (SPLIT ? p * NP + v : p)) * 3 + c) * NZ + z] = o;
            }
        named_bar_sync(1, Cfg::NC);
        for (int o = tid; o < B * PTS * 3 * NZ; o += Cfg::NC) {
            const int bb = o / (PTS * 3 * NZ), rem = o - bb * PTS * 3 * NZ, p = rem / (3 * NZ) / NP;
            C2 v = red[bb * PTS * 3 * NZ + rem];
#pragma unroll
            for (int ss = 1; ss < S; ss++) {
                const C2 w = red[(ss * B + bb) * PTS * 3 * NZ + rem];
                v.x += w.x;
                v.y += w.y;
            }
            const long long unit = batch * B + bb;
            const int q = (int)(unit / Ny), r = (int)(unit - (long long)q * Ny);
            if ((q == 0 && (p & 2)) || (r == 0 && (p & 1))) { v.x = R(0); v.y = R(0); }
            Uhat[unit * PTS * Cfg::Z3 + rem] = v;
        }
        named_bar_sync(1, Cfg::NC);  // red reads done before the slot is refilled
        mbar_arrive(&empty[slot]);
    }
}

// ------------------------------------------------------------------------------------------------
// Barrier-free form: the j-slices of a row sit in one warp and are reduced with shuffles.
//
// Threads (g, w, lane): warp group g takes the CTA's units (tickets) it = g, g + NG, ...; warp w of the
// group owns rows z = w*ZW + zl, and lane = zl + ZW*s sums j = s, s + SL, s + 2 SL, ... (interleaved
// slices: the SL lanes of one zl read SL consecutive spectrum entries, one wavefront).  Ticket it uses
// stage it % NSTAGE in round it / NSTAGE.  A parity wait cannot tell round r from round r-2, and with
// several groups on one ring a group could reach round r of a stage while round r-1 (another group's
// ticket) is still in flight.  So tickets are passed in order: a warp starts waiting for ticket it only
// once ticket it-1 has been passed (a shared counter raised with atomicMax), which by induction means
// round r-1 of its stage has landed and the parity wait is exact.  After its last shared-memory read
// every lane arrives on the stage's empty barrier (it counts the group's threads), so the producer
// refills the stage while the warp reduces.  The reduction is a recursive halving over the lane bits of
// s: each step sends half of the outputs a lane still holds to its partner and adds the half it
// receives, so every lane ends with NR/SL of the NR = 2*3*PTS reals and stores them.  No CTA-wide
// barrier is left in the consumer loop: one warp's reduction and stores overlap another's FMAs.
template <typename R, int NZ, int SL, int NG, int NSTAGE, int NP, int MINB, int VS = 1>
struct CfgL {
    static constexpr int P = NZ * (NZ + 1) / 2;
    static constexpr int T = 4 * P + 2 * NZ * NZ;
    static constexpr int Z3 = 3 * NZ;
    static constexpr int PTS = 4 * NP;
    static constexpr int PL = LanePts<NP, VS>::PL;  // points per lane
    static constexpr int ZW = 32 / (SL * VS);      // rows per warp
    static constexpr int W = NZ / ZW;    // warps per group
    static constexpr int NC = NG * W * 32;
    static constexpr int NTHREADS = NC + 32;
    static constexpr int JS = NZ / SL;
    static constexpr int ES = 2 * sizeof(R);
    static constexpr int TBYTES = T * ES;
    static constexpr int UBYTES = PTS * Z3 * ES;
    static constexpr int STAGE_BYTES = TBYTES + UBYTES;
    static constexpr int NR = 2 * 3 * PL;   // reals per lane before the reduction
    static constexpr int HR = NR / SL;      // reals per lane after it
    static constexpr int SMEM = NSTAGE * STAGE_BYTES + 2 * NSTAGE * 8 + 16;  // + ticket counter
    static_assert(32 % (SL * VS) == 0 && NZ % ZW == 0, "slices x vector groups must tile a warp, warps the rows");
    static_assert(NR % SL == 0 && HR % 2 == 0, "every lane must end with whole complex outputs");
    static_assert(STAGE_BYTES % 16 == 0 && TBYTES % 16 == 0, "bulk copies need 16-byte multiples");
    static_assert(SMEM <= 232448, "exceeds the 227 KB dynamic shared memory of one CTA");
    static_assert(MINB * (SMEM + 1024) <= 233472, "MINB CTAs do not fit the SM's shared memory");
};

// PK (complex64): the packed 3-multiply form of k_contract_tma, two instructions per complex multiply-add.
// VS: the NP vectors of a unit split over VS lane groups (LanePts): fewer points and registers per lane.
// UR: j iterations of the unit sums unrolled together (wl_unit_sums)
template <typename R, int NZ, int SL, int NG, int NSTAGE, int NP, int MINB, bool M4, bool PK, int VS = 1, int UR = 2>
__global__ void __launch_bounds__(CfgL<R, NZ, SL, NG, NSTAGE, NP, MINB, VS>::NTHREADS, MINB)
    k_contract_wl(const typename V2<R>::T *__restrict__ G, typename V2<R>::T *__restrict__ Uhat, int Ny,
                  long long nunits, int *err, const int *gate)
{
    if (gate && *gate == 0) return;  // uniform across the CTA: nothing has been issued yet
    using Cfg = CfgL<R, NZ, SL, NG, NSTAGE, NP, MINB, VS>;
    constexpr int PTS = Cfg::PTS, ZW = Cfg::ZW, W = Cfg::W;
    using C2 = typename V2<R>::T;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *stages = smem;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + NSTAGE * Cfg::STAGE_BYTES);
    uint64_t *empty = full + NSTAGE;
    int *passed = reinterpret_cast<int *>(empty + NSTAGE);  // tickets [0, *passed) have been passed

    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], W * 32);
        }
        *passed = 0;
        fence_mbar_init();
    }
    __syncthreads();

    const long long first = blockIdx.x, stride = gridDim.x;
    const long long my_n = first < nunits ? (nunits - 1 - first) / stride + 1 : 0;

    if (tid >= Cfg::NC) {
        // producer warp: one lane streams units (tensor + 4-point spectra) into the stage ring in order
        if (tid == Cfg::NC) {
            const uint64_t pol_t = l2_policy_evict_first();
            const uint64_t pol_u = l2_policy_evict_normal();
            long long issued = 0;
            bool ok = true;
            for (long long it = 0; it < my_n; it++) {
                const int slot = (int)(it % NSTAGE);
                const uint32_t round = (uint32_t)(it / NSTAGE);
                if (round > 0) {
                    if (!mbar_wait_bounded(&empty[slot], (round - 1) & 1, err, 14)) { ok = false; break; }
                }
                const long long unit = first + it * stride;
                unsigned char *st = stages + slot * Cfg::STAGE_BYTES;
                mbar_arrive_expect_tx(&full[slot], Cfg::STAGE_BYTES);
                bulk_g2s(st, G + unit * (long long)Cfg::T, Cfg::TBYTES, &full[slot], pol_t);
                bulk_g2s(st + Cfg::TBYTES, Uhat + unit * (long long)PTS * Cfg::Z3, Cfg::UBYTES, &full[slot], pol_u);
                issued++;
            }
            if (!ok) {
                for (long long it = (issued > NSTAGE ? issued - NSTAGE : 0); it < issued; it++)
                    mbar_wait_bounded(&full[it % NSTAGE], (uint32_t)(it / NSTAGE) & 1, err, 16);
            }
        }
        return;
    }

    const int warp = tid >> 5, lane = tid & 31;
    const int g = warp / W, z = (warp % W) * ZW + lane % ZW, s = (lane / ZW) % SL, vv = lane / (ZW * SL);
    for (long long it = g; it < my_n; it += NG) {
        const int slot = (int)(it % NSTAGE);
        const uint32_t round = (uint32_t)(it / NSTAGE);
        // the warp leaves together (its lanes shuffle with one another below)
        if (!__all_sync(0xffffffffu, wait_ticket(passed, (int)it, err))) return;
        __threadfence_block();
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full[slot], round & 1, err, 15))) return;
        __threadfence_block();
        if (lane == 0) atomicMax(passed, (int)it + 1);
        const unsigned char *st = stages + slot * Cfg::STAGE_BYTES;
        const C2 *gb = reinterpret_cast<const C2 *>(st);
        const C2 *ub = reinterpret_cast<const C2 *>(st + Cfg::TBYTES);  // [pt][c][j]
        R v[Cfg::NR];
        wl_unit_sums<R, NZ, SL, NP, M4, PK, VS, UR>(gb, ub, z, s, v, vv);
        mbar_arrive(&empty[slot]);  // this lane's reads of the stage are done

        const long long unit = first + it * stride;
        const int q = (int)(unit / Ny), r = (int)(unit - (long long)q * Ny);
        wl_unit_store<R, NZ, SL, NP, VS>(v, s, q, r, Uhat + unit * PTS * Cfg::Z3 + z, vv);
    }
}

// ------------------------------------------------------------------------------------------------
// complex64 contraction in the Walsh basis of the four points, with packed FP32 pair arithmetic.
//
// The four points of a unit, p = (sx bit, m bit), form the group Z2 x Z2 and every term of the sign table
// carries one of its characters chi_t(p) = (-1)^popc(t & p): t = 0 for xx, yy, zz, t = 3 for xy (sx m),
// t = 2 for xz and zx (sx), t = 1 for yz and zy (m), with a fixed minus on zx and zy.  In the Walsh basis
// U^[w] = sum_p chi_w(p) U[p] a character becomes an index shift, so
//     out^[C][w] = sum_terms (+-) G_term U^[IN][w xor t],   out[p] = 1/4 sum_w chi_w(p) out^[w]:
// no per-point signs remain in the inner loop.  Each complex multiply-add is two fma.rn.f32x2:
//     acc1 += (g.x, g.y) * (u.x, u.x),   acc2 += (g.x, g.y) * (u.y, u.y)
//     -> re = acc1.x - acc2.y,  im = acc1.y + acc2.x,
// with the broadcast pairs (u.x, u.x), (u.y, u.y) prepared once per unit in shared memory.  Per j a thread
// issues 8 tensor loads, 24 broadcast loads and 72 packed FMAs (144 FMAs).
// Threads (b, v, s, z): unit b of the stage, vector v (NP vectors share the tensor), j-slice s, row z.
template <int NZ, int S, int B, int NSTAGE, int NP, int MINB = 1>
struct CfgW {
    static constexpr int P = NZ * (NZ + 1) / 2;
    static constexpr int T = 4 * P + 2 * NZ * NZ;
    static constexpr int Z3 = 3 * NZ;
    static constexpr int PTS = 4 * NP;
    static constexpr int NC = B * NP * S * NZ;
    static constexpr int NTHREADS = NC + 32;
    static constexpr int JS = NZ / S;
    static constexpr int TBYTES = B * T * 8;
    static constexpr int UBYTES = B * PTS * Z3 * 8;
    static constexpr int STAGE_BYTES = TBYTES + UBYTES;
    static constexpr int UE_BYTES = B * NP * 3 * 4 * NZ * 16;  // broadcast pairs of the Walsh spectra
    static constexpr int RED_BYTES = S * B * NP * 12 * NZ * 8;
    static constexpr int SMEM = NSTAGE * STAGE_BYTES + UE_BYTES + 2 * NSTAGE * 8 + 16;
    static_assert(NZ % S == 0, "slices must divide Nz");
    static_assert(NC % 32 == 0, "consumer threads must be whole warps");
    static_assert(RED_BYTES <= TBYTES, "reduction buffer reuses the drained tensor stage");
    static_assert(STAGE_BYTES % 16 == 0 && TBYTES % 16 == 0, "bulk copies need 16-byte multiples");
    static_assert(SMEM <= 232448, "exceeds the 227 KB dynamic shared memory of one CTA");
    static_assert(MINB * (SMEM + 1024) <= 233472, "MINB CTAs do not fit the SM's shared memory");
};

template <int NZ, int S, int B, int NSTAGE, int NP, int MINB>
__global__ void __launch_bounds__(CfgW<NZ, S, B, NSTAGE, NP, MINB>::NTHREADS, MINB)
    k_contract_w32(const float2 *__restrict__ G, float2 *__restrict__ Uhat, int Ny, long long nbatches, int *err,
                   const int *gate)
{
    if (gate && *gate == 0) return;
    using Cfg = CfgW<NZ, S, B, NSTAGE, NP, MINB>;
    constexpr int PTS = Cfg::PTS, Z3 = Cfg::Z3;
    constexpr int AW = asw_width32(NZ);
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *stages = smem;
    float2 *ue = reinterpret_cast<float2 *>(smem + NSTAGE * Cfg::STAGE_BYTES);  // [b][v][c][w][j][2]
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + NSTAGE * Cfg::STAGE_BYTES + Cfg::UE_BYTES);
    uint64_t *empty = full + NSTAGE;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + NSTAGE);

    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], Cfg::NC);
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    const long long first = blockIdx.x, stride = gridDim.x;
    const long long my_n = first < nbatches ? (nbatches - 1 - first) / stride + 1 : 0;

    if (tid >= Cfg::NC) {
        // producer warp: one lane streams tensor units and their spectra into the stage ring
        if (tid == Cfg::NC) {
            const uint64_t pol_t = l2_policy_evict_first();
            const uint64_t pol_u = l2_policy_evict_normal();
            long long issued = 0;
            bool ok = true;
            for (long long it = 0; it < my_n; it++) {
                const int slot = (int)(it % NSTAGE);
                const uint32_t round = (uint32_t)(it / NSTAGE);
                if (it >= NSTAGE) {
                    if (!mbar_wait_bounded(&empty[slot], (round - 1) & 1, err, 21)) { ok = false; break; }
                }
                const long long batch = first + it * stride;
                unsigned char *st = stages + slot * Cfg::STAGE_BYTES;
                mbar_arrive_expect_tx(&full[slot], Cfg::STAGE_BYTES);
                bulk_g2s(st, G + batch * (long long)B * Cfg::T, Cfg::TBYTES, &full[slot], pol_t);
                bulk_g2s(st + Cfg::TBYTES, Uhat + batch * (long long)B * PTS * Z3, Cfg::UBYTES, &full[slot], pol_u);
                issued++;
            }
            if (!ok) {
                for (long long it = (issued > NSTAGE ? issued - NSTAGE : 0); it < issued; it++)
                    mbar_wait_bounded(&full[it % NSTAGE], (uint32_t)(it / NSTAGE) & 1, err, 22);
            }
        }
        return;
    }

    const int z = tid % NZ;
    const int s = (tid / NZ) % S;
    const int v = (tid / (NZ * S)) % NP;
    const int b = tid / (NZ * S * NP);
    for (long long it = 0; it < my_n; it++) {
        const int slot = (int)(it % NSTAGE);
        const uint32_t round = (uint32_t)(it / NSTAGE);
        const bool ok = mbar_wait_bounded(&full[slot], round & 1, err, 23);
        if (!ok) *abort_flag = 1;
        const long long batch = first + it * stride;
        unsigned char *st = stages + slot * Cfg::STAGE_BYTES;
        const float2 *gt = reinterpret_cast<const float2 *>(st);
        const float2 *uh = reinterpret_cast<const float2 *>(st + Cfg::TBYTES);  // [b][slot][v][c][j]
        if (ok) {
            // Walsh transform over the 4 points and broadcast pairs: ue[b][v][c][w][j] = {(x,x), (y,y)}
            for (int o = tid; o < B * NP * 3 * NZ; o += Cfg::NC) {
                const int jj = o % NZ, c = (o / NZ) % 3, vv = (o / Z3) % NP, bb = o / (Z3 * NP);
                float2 u[4];
#pragma unroll
                for (int p = 0; p < 4; p++) u[p] = uh[((bb * 4 + p) * NP + vv) * Z3 + c * NZ + jj];
                const float2 a0 = make_float2(u[0].x + u[1].x, u[0].y + u[1].y);
                const float2 a1 = make_float2(u[0].x - u[1].x, u[0].y - u[1].y);
                const float2 a2 = make_float2(u[2].x + u[3].x, u[2].y + u[3].y);
                const float2 a3 = make_float2(u[2].x - u[3].x, u[2].y - u[3].y);
                const float2 w4[4] = {make_float2(a0.x + a2.x, a0.y + a2.y), make_float2(a1.x + a3.x, a1.y + a3.y),
                                      make_float2(a0.x - a2.x, a0.y - a2.y), make_float2(a1.x - a3.x, a1.y - a3.y)};
                float2 *dst = ue + ((bb * NP + vv) * 3 + c) * 4 * NZ * 2;
#pragma unroll
                for (int w = 0; w < 4; w++) {
                    dst[(w * NZ + jj) * 2 + 0] = make_float2(w4[w].x, w4[w].x);
                    dst[(w * NZ + jj) * 2 + 1] = make_float2(w4[w].y, w4[w].y);
                }
            }
        }
        named_bar_sync(1, Cfg::NC);  // Walsh pairs ready (or the wait gave up everywhere)
        if (*abort_flag) return;

        float2 acc1[3][4], acc2[3][4];
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int w = 0; w < 4; w++) acc1[c][w] = acc2[c][w] = make_float2(0.f, 0.f);
        const float2 *gb = gt + b * Cfg::T;
        const float2 *gxx = gb, *gxy = gb + Cfg::P, *gyy = gb + 2 * Cfg::P, *gzz = gb + 3 * Cfg::P;
        const float2 *gxz = gb + 4 * Cfg::P, *gyz = gb + 4 * Cfg::P + NZ * NZ;
        const float2 *ub = ue + (b * NP + v) * 3 * 4 * NZ * 2;
#pragma unroll 1
        for (int jj = 0; jj < Cfg::JS; jj++) {
            const int j = s * Cfg::JS + jj;
            const int si = sym_idx<NZ>(z, j);
            const int a_zj = asw(z, j, NZ, AW), a_jz = asw(j, z, NZ, AW);
            const float2 exx = gxx[si], exy = gxy[si], eyy = gyy[si], ezz = gzz[si];
            const float2 exz = gxz[a_zj], eyz = gyz[a_zj];
            const float2 ezx = make_float2(-gxz[a_jz].x, -gxz[a_jz].y);  // -xz^T
            const float2 ezy = make_float2(-gyz[a_jz].x, -gyz[a_jz].y);  // -yz^T
#pragma unroll
            for (int wi = 0; wi < 4; wi++) {
                // input x at Walsh index wi feeds out x (xx, t=0), out y (xy, t=3), out z (-zx, t=2)
                const float2 px = ub[((0 * 4 + wi) * NZ + j) * 2 + 0], py = ub[((0 * 4 + wi) * NZ + j) * 2 + 1];
                acc1[0][wi] = ffma2(exx, px, acc1[0][wi]);
                acc2[0][wi] = ffma2(exx, py, acc2[0][wi]);
                acc1[1][wi ^ 3] = ffma2(exy, px, acc1[1][wi ^ 3]);
                acc2[1][wi ^ 3] = ffma2(exy, py, acc2[1][wi ^ 3]);
                acc1[2][wi ^ 2] = ffma2(ezx, px, acc1[2][wi ^ 2]);
                acc2[2][wi ^ 2] = ffma2(ezx, py, acc2[2][wi ^ 2]);
            }
#pragma unroll
            for (int wi = 0; wi < 4; wi++) {
                // input y: out x (xy, t=3), out y (yy, t=0), out z (-zy, t=1)
                const float2 px = ub[((1 * 4 + wi) * NZ + j) * 2 + 0], py = ub[((1 * 4 + wi) * NZ + j) * 2 + 1];
                acc1[0][wi ^ 3] = ffma2(exy, px, acc1[0][wi ^ 3]);
                acc2[0][wi ^ 3] = ffma2(exy, py, acc2[0][wi ^ 3]);
                acc1[1][wi] = ffma2(eyy, px, acc1[1][wi]);
                acc2[1][wi] = ffma2(eyy, py, acc2[1][wi]);
                acc1[2][wi ^ 1] = ffma2(ezy, px, acc1[2][wi ^ 1]);
                acc2[2][wi ^ 1] = ffma2(ezy, py, acc2[2][wi ^ 1]);
            }
#pragma unroll
            for (int wi = 0; wi < 4; wi++) {
                // input z: out x (xz, t=2), out y (yz, t=1), out z (zz, t=0)
                const float2 px = ub[((2 * 4 + wi) * NZ + j) * 2 + 0], py = ub[((2 * 4 + wi) * NZ + j) * 2 + 1];
                acc1[0][wi ^ 2] = ffma2(exz, px, acc1[0][wi ^ 2]);
                acc2[0][wi ^ 2] = ffma2(exz, py, acc2[0][wi ^ 2]);
                acc1[1][wi ^ 1] = ffma2(eyz, px, acc1[1][wi ^ 1]);
                acc2[1][wi ^ 1] = ffma2(eyz, py, acc2[1][wi ^ 1]);
                acc1[2][wi] = ffma2(ezz, px, acc1[2][wi]);
                acc2[2][wi] = ffma2(ezz, py, acc2[2][wi]);
            }
        }
        named_bar_sync(1, Cfg::NC);  // every read of this stage's tensor is done
        // slice partials of the Walsh outputs into the drained tensor area: red[s][b][v][c][w][z]
        float2 *red = reinterpret_cast<float2 *>(st);
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int w = 0; w < 4; w++)
                red[((((s * B + b) * NP + v) * 3 + c) * 4 + w) * NZ + z] =
                    make_float2(acc1[c][w].x - acc2[c][w].y, acc1[c][w].y + acc2[c][w].x);
        named_bar_sync(1, Cfg::NC);
        for (int o = tid; o < B * NP * 3 * NZ; o += Cfg::NC) {
            const int zz = o % NZ, c = (o / NZ) % 3, vv = (o / Z3) % NP, bb = o / (Z3 * NP);
            float2 h[4];
#pragma unroll
            for (int w = 0; w < 4; w++) {
                float2 t = red[((((0 * B + bb) * NP + vv) * 3 + c) * 4 + w) * NZ + zz];
#pragma unroll
                for (int ss = 1; ss < S; ss++) {
                    const float2 q = red[((((ss * B + bb) * NP + vv) * 3 + c) * 4 + w) * NZ + zz];
                    t.x += q.x;
                    t.y += q.y;
                }
                h[w] = t;
            }
            // inverse Walsh transform, 1/4 exact
            const float2 a0 = make_float2(h[0].x + h[1].x, h[0].y + h[1].y);
            const float2 a1 = make_float2(h[0].x - h[1].x, h[0].y - h[1].y);
            const float2 a2 = make_float2(h[2].x + h[3].x, h[2].y + h[3].y);
            const float2 a3 = make_float2(h[2].x - h[3].x, h[2].y - h[3].y);
            float2 outp[4] = {make_float2(0.25f * (a0.x + a2.x), 0.25f * (a0.y + a2.y)),
                              make_float2(0.25f * (a1.x + a3.x), 0.25f * (a1.y + a3.y)),
                              make_float2(0.25f * (a0.x - a2.x), 0.25f * (a0.y - a2.y)),
                              make_float2(0.25f * (a1.x - a3.x), 0.25f * (a1.y - a3.y))};
            const long long unit = batch * B + bb;
            const int q = (int)(unit / Ny), r = (int)(unit - (long long)q * Ny);
#pragma unroll
            for (int p = 0; p < 4; p++) {
                if ((q == 0 && (p & 2)) || (r == 0 && (p & 1))) outp[p] = make_float2(0.f, 0.f);
                Uhat[unit * PTS * Z3 + (p * NP + vv) * Z3 + c * NZ + zz] = outp[p];
            }
        }
        named_bar_sync(1, Cfg::NC);  // red reads done before the slot is refilled
        mbar_arrive(&empty[slot]);
    }
}

template <int NZ, int S, int B, int NSTAGE, int NP, int MINB = 1>
int launch_w32(const float2 *G, float2 *Uhat, int Nx, int Ny, int *err, int nsm, cudaStream_t st, const int *gate)
{
    using Cfg = CfgW<NZ, S, B, NSTAGE, NP, MINB>;
    auto kern = k_contract_w32<NZ, S, B, NSTAGE, NP, MINB>;
    nsm *= MINB;
    static bool attr = false;
    if (!attr) {
        G2_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
        attr = true;
    }
    const long long units = (long long)Nx * Ny;
    if (units % B) return G2_ERR_UNSUPPORTED;
    const long long nb = units / B;
    const int grid = (int)(nb < nsm ? nb : nsm);
    kern<<<grid, Cfg::NTHREADS, Cfg::SMEM, st>>>(G, Uhat, Ny, nb, err, gate);
    G2_CUDA_CHECK(cudaGetLastError());
    return G2_OK;
}

// MINB CTAs per SM: their compute, reduction and barrier phases overlap one another
template <typename R, int NZ, int S, int B, int NSTAGE, int NP = 1, bool SPLIT = false, int MINB = 1, bool M4 = false,
          bool PK = false>
int launch_cfg(const void *G, void *Uhat, int Nx, int Ny, int *err, int nsm, cudaStream_t st, const int *gate)
{
    using Cfg = CfgT<R, NZ, S, B, NSTAGE, NP, SPLIT, MINB>;
    auto kern = k_contract_tma<R, NZ, S, B, NSTAGE, NP, SPLIT, MINB, M4, PK>;
    nsm *= MINB;
    static bool attr = false;
    if (!attr) {
        G2_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
        attr = true;
    }
    const long long units = (long long)Nx * Ny;
    if (units % B) return G2_ERR_UNSUPPORTED;
    const long long nb = units / B;
    const int grid = (int)(nb < nsm ? nb : nsm);
    kern<<<grid, Cfg::NTHREADS, Cfg::SMEM, st>>>(reinterpret_cast<const typename V2<R>::T *>(G),
                                                 reinterpret_cast<typename V2<R>::T *>(Uhat), Ny, nb, err, gate);
    G2_CUDA_CHECK(cudaGetLastError());
    return G2_OK;
}

template <typename R, int NZ, int SL, int NG, int NSTAGE, int NP = 1, int MINB = 1, bool M4 = false, bool PK = false,
          int VS = 1, int UR = 2>
int launch_wl(const void *G, void *Uhat, int Nx, int Ny, int *err, int nsm, cudaStream_t st, const int *gate)
{
    using Cfg = CfgL<R, NZ, SL, NG, NSTAGE, NP, MINB, VS>;
    auto kern = k_contract_wl<R, NZ, SL, NG, NSTAGE, NP, MINB, M4, PK, VS, UR>;
    nsm *= MINB;
    static bool attr = false;
    if (!attr) {
        G2_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
        attr = true;
    }
    const long long units = (long long)Nx * Ny;
    const int grid = (int)(units < nsm ? units : nsm);
    kern<<<grid, Cfg::NTHREADS, Cfg::SMEM, st>>>(reinterpret_cast<const typename V2<R>::T *>(G),
                                                 reinterpret_cast<typename V2<R>::T *>(Uhat), Ny, units, err, gate);
    G2_CUDA_CHECK(cudaGetLastError());
    return G2_OK;
}

int sm_count()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    }
    return n;
}

}  // namespace

// Tile-shape variants per (precision, Nz); variant 0 is the default.  The autotuner times the variants
// on the operator's own buffers and stores its pick in the operator.
int ie_contract_variants(int precision, int Nz)
{
    if (precision == 0) return Nz == 32 ? 12 : (Nz == 8 || Nz == 16 || Nz == 48 ? 2 : 0);
    return Nz == 32 ? 25 : (Nz == 8 || Nz == 16 || Nz == 48 ? 4 : 0);
}

// Returns G2_ERR_UNSUPPORTED when no specialised configuration exists (caller uses the generic kernel).
int ie_contract_fast64(const double2 *G, double2 *Uhat, int Nx, int Ny, int Nz, int *err, cudaStream_t st, int v,
                       const int *gate)
{
    const int n = sm_count();
    switch (Nz) {
    case 8:
        if (v == 1) return launch_wl<double, 8, 4, 8, 16>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<double, 8, 2, 8, 4>(G, Uhat, Nx, Ny, err, n, st, gate);
    case 16:
        if (v == 1) return launch_wl<double, 16, 4, 4, 8>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<double, 16, 4, 4, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
    case 48:
        if (v == 1) return launch_wl<double, 48, 4, 1, 1>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<double, 48, 4, 1, 1>(G, Uhat, Nx, Ny, err, n, st, gate);
    case 32:
        if (v == 1) return launch_cfg<double, 32, 4, 1, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 2) return launch_cfg<double, 32, 4, 1, 1, 1, false, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 3) return launch_cfg<double, 32, 2, 1, 1, 1, false, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 4) return launch_cfg<double, 32, 4, 1, 1, 1, false, 3, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 5) return launch_wl<double, 32, 4, 2, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 6) return launch_wl<double, 32, 4, 3, 3, 1, 1, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 7) return launch_wl<double, 32, 4, 1, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 8) return launch_wl<double, 32, 2, 3, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 9) return launch_wl<double, 32, 2, 4, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 10) return launch_wl<double, 32, 4, 2, 3, 1, 1, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 11) return launch_wl<double, 32, 4, 2, 3, 1, 1, false, false, 1, 4>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<double, 32, 8, 1, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
    default: return G2_ERR_UNSUPPORTED;
    }
}
// complex64 variants: the direct kernel (k_contract_tma) and the Walsh-basis packed kernel (k_contract_w32)
int ie_contract_fast32(const float2 *G, float2 *Uhat, int Nx, int Ny, int Nz, int *err, cudaStream_t st, int v,
                       const int *gate)
{
    const int n = sm_count();
    switch (Nz) {
    case 8:
        if (v == 1) return launch_w32<8, 2, 16, 3, 1>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 2) return launch_wl<float, 8, 4, 8, 16>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 3) return launch_wl<float, 8, 4, 8, 16, 1, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<float, 8, 2, 16, 4>(G, Uhat, Nx, Ny, err, n, st, gate);
    case 16:
        if (v == 1) return launch_w32<16, 4, 4, 4, 1>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 2) return launch_wl<float, 16, 2, 8, 8>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 3) return launch_wl<float, 16, 2, 8, 8, 1, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<float, 16, 4, 4, 4>(G, Uhat, Nx, Ny, err, n, st, gate);
    case 32:
        switch (v) {
        case 1: return launch_cfg<float, 32, 4, 1, 5>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 2: return launch_cfg<float, 32, 8, 2, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 3: return launch_w32<32, 8, 1, 5, 1>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 4: return launch_w32<32, 8, 2, 2, 1>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 5: return launch_w32<32, 4, 2, 2, 1>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 6: return launch_cfg<float, 32, 8, 1, 3, 1, false, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 7: return launch_cfg<float, 32, 4, 1, 3, 1, false, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 8: return launch_cfg<float, 32, 4, 1, 2, 1, false, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 9: return launch_cfg<float, 32, 2, 1, 1, 1, false, 6>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 10: return launch_cfg<float, 32, 2, 1, 2, 1, false, 3>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 11: return launch_w32<32, 4, 1, 2, 1, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 12: return launch_cfg<float, 32, 4, 1, 2, 1, false, 3, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 13: return launch_cfg<float, 32, 4, 1, 3, 1, false, 2, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 14: return launch_wl<float, 32, 4, 3, 6>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 15: return launch_wl<float, 32, 4, 2, 6>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 16: return launch_wl<float, 32, 2, 4, 6>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 17: return launch_wl<float, 32, 4, 4, 6>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 18: return launch_wl<float, 32, 2, 6, 6>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 19: return launch_wl<float, 32, 2, 5, 6>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 20: return launch_wl<float, 32, 1, 8, 6>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 21: return launch_wl<float, 32, 2, 6, 6, 1, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 22: return launch_wl<float, 32, 2, 4, 6, 1, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 23: return launch_wl<float, 32, 4, 4, 6, 1, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        case 24: return launch_wl<float, 32, 2, 6, 6, 1, 1, false, true, 1, 4>(G, Uhat, Nx, Ny, err, n, st, gate);
        default: return launch_cfg<float, 32, 8, 1, 5>(G, Uhat, Nx, Ny, err, n, st, gate);
        }
    case 48:
        if (v == 1) return launch_w32<48, 4, 1, 2, 1>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 2) return launch_wl<float, 48, 4, 2, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 3) return launch_wl<float, 48, 4, 2, 2, 1, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<float, 48, 4, 1, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
    default: return G2_ERR_UNSUPPORTED;
    }
}

// Two vectors of one operator per tensor read (complex64; both polarisations of a plane-wave source).
// The spectrum holds [unit][slot][vector][3Nz].  Variants: 0 the direct kernel with the two vectors spread
// over threads, 1 the direct kernel with both vectors in each thread's registers, 2 (and 3) the
// Walsh-basis packed kernel.
int ie_contract_pair_variants(int Nz) { return Nz == 32 ? 21 : (Nz == 48 ? 6 : ((Nz == 8 || Nz == 16) ? 4 : 0)); }
int ie_contract_pair32(const float2 *G, float2 *Uhat, int Nx, int Ny, int Nz, int *err, cudaStream_t st,
                       const int *gate, int v)
{
    const int n = sm_count();
    switch (Nz) {
    case 8:
        if (v == 1) return launch_cfg<float, 8, 1, 16, 3, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 2) return launch_w32<8, 1, 16, 2, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 3) return launch_wl<float, 8, 4, 8, 16, 2, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<float, 8, 1, 16, 3, 2, true>(G, Uhat, Nx, Ny, err, n, st, gate);
    case 16:
        if (v == 1) return launch_cfg<float, 16, 2, 4, 4, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 2) return launch_w32<16, 2, 4, 4, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 3) return launch_wl<float, 16, 2, 4, 8, 2, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<float, 16, 2, 4, 4, 2, true>(G, Uhat, Nx, Ny, err, n, st, gate);
    case 32:
        if (v == 1) return launch_cfg<float, 32, 4, 1, 5, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 2) return launch_w32<32, 4, 2, 2, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 3) return launch_w32<32, 4, 1, 5, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 4) return launch_cfg<float, 32, 4, 1, 2, 2, true, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 5) return launch_cfg<float, 32, 4, 1, 2, 2, false, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 6) return launch_cfg<float, 32, 2, 1, 1, 2, true, 4>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 7) return launch_w32<32, 4, 1, 2, 2, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 8) return launch_cfg<float, 32, 4, 1, 2, 2, false, 2, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 9) return launch_wl<float, 32, 4, 2, 5, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 10) return launch_wl<float, 32, 8, 1, 5, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 11) return launch_wl<float, 32, 2, 4, 5, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 12) return launch_wl<float, 32, 2, 5, 5, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 13) return launch_wl<float, 32, 2, 3, 5, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 14) return launch_wl<float, 32, 2, 4, 5, 2, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 15) return launch_wl<float, 32, 2, 5, 5, 2, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        // the two vectors split over lane groups: 4 points per lane
        if (v == 16) return launch_wl<float, 32, 2, 3, 5, 2, 1, false, true, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 17) return launch_wl<float, 32, 2, 4, 5, 2, 1, false, true, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 18) return launch_wl<float, 32, 2, 2, 5, 2, 1, false, true, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 19) return launch_wl<float, 32, 4, 2, 5, 2, 1, false, true, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        // variant 14 with four j iterations unrolled together
        if (v == 20) return launch_wl<float, 32, 2, 4, 5, 2, 1, false, true, 1, 4>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<float, 32, 4, 2, 2, 2, true>(G, Uhat, Nx, Ny, err, n, st, gate);
    case 48:
        if (v == 1) return launch_cfg<float, 48, 4, 1, 2, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 2) return launch_w32<48, 4, 1, 2, 2>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 3) return launch_wl<float, 48, 4, 1, 2, 2, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        // two consumer groups, or eight j-slices per row: 1.86 / 1.90 ms against 2.37 ms for variant 3 at
        // 256x256x48 (standalone timing of the contraction alone)
        if (v == 4) return launch_wl<float, 48, 4, 2, 2, 2, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        if (v == 5) return launch_wl<float, 48, 8, 1, 2, 2, 1, false, true>(G, Uhat, Nx, Ny, err, n, st, gate);
        return launch_cfg<float, 48, 4, 1, 2, 2, true>(G, Uhat, Nx, Ny, err, n, st, gate);
    default: return G2_ERR_UNSUPPORTED;
    }
}
bool ie_contract_pair32_supported(int Nx, int Ny, int Nz)
{
    const long long u = (long long)Nx * Ny;
    switch (Nz) {
    case 8: return u % 16 == 0;
    case 16: return u % 4 == 0;
    case 32:
    case 48: return true;
    default: return false;
    }
}
