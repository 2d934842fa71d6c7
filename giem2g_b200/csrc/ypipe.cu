// The y-transforms fused with the Green's-tensor contraction: one persistent kernel in place of
// k_fy -> contraction -> k_by (apply.cu), so the 2-D spectrum never makes a round trip through HBM.  It is
// a tile-shape variant (giem2g_set_contract_variant, the last two of each form at Nz = 32), not the default:
// measured on a B200 at 128x128x32 the separate passes are faster (FP64 apply 0.33 against 0.47 ms).  Three
// FFT warps per SM need about 0.1 ms for the y-transforms of one apply on their own, and the FP64 stage
// ring has room for two stages beside the transform lines, so the pass costs about what the spectrum's round
// trip saves (both roles timed apart in a probe: FP64 contraction role 0.26-0.29 ms, FFT role 0.16 ms;
// complex64 0.12 and 0.10 ms; the separate k_fy + contraction + k_by take 0.27 and 0.17 ms).
//
// Restates the middle of MULT_IE_OP (apply_ie_operator_module.F90:189-263): the forward y-FFT with its +-ky
// repack (Distributed_FFT.F90:437-505), VERTICAL_MULT_GENERAL at every (kx-pair, ky-pair) unit
// (apply_ie_operator_module.F90:265-374), and the inverse y-FFT with its repack (Distributed_FFT.F90:696-788).
//
// Why one kernel.  Between the passes the spectrum of the whole grid (4x the vector: 100 MB in FP64 at
// 128x128x32) went to HBM and back three times.  Here the kx pairs are processed in batches of kQB pairs,
// so only a few batches of spectrum are alive at a time (a few MB), and they stay in the 126 MB L2.
//
// Why not thread-block clusters.  Holding one kx pair's spectrum in distributed shared memory takes an
// 8-CTA cluster at ~226 KB per CTA, and a B200 keeps only 15 such clusters resident (120 of 148 SMs;
// 33 clusters of 4 = 132 SMs).  This kernel runs one CTA on every SM instead and exchanges through L2.
//
// Roles (warp-specialised, one CTA per SM, no CTA-wide barrier after the start):
//   * producer warp (one lane): grabs the next unit from a global counter, streams its tensor
//     (cp.async.bulk, L2 evict_first) into a stage of the ring at once, waits until the forward
//     transforms of the unit's batch are complete, then streams the unit's four spectral points
//     (L2-resident) into the same stage;
//   * consumer warps: the barrier-free contraction of contract_wl.cuh (warp groups taking stage tickets
//     in order), outputs written back in place into the spectrum; every warp counts its finished units
//     into the batch's completion counter;
//   * FFT warps: grab transform tasks in a fixed order -- forward tasks of batch 0, 1, then inverse of
//     batch b-1 after forward of batch b, ..., inverse of the last batch -- each the y-FFT of NL lines of
//     one kx column (the four-step register FFT of fft4.cuh, the same arithmetic as k_fy / k_by).  An
//     inverse task waits until its batch's units are all contracted; it reads the spectrum with L2-only
//     loads (L1 is not coherent across SMs) and writes the cropped result into U1 for k_bx.
// Every wait is bounded (2 s): on timeout the kernel records a code in the device error word and carries
// on, so every role still reaches its end (the result is then invalid and the host reports the code).
// No role depends on another CTA being resident: work is grabbed only by running CTAs and every wait is
// for work grabbed earlier (forward tasks of a batch precede every inverse task that could block an FFT
// warp; units are grabbed in batch order), so the pipeline cannot deadlock.
//
// The x-Nyquist column (kx = Nx, kx-pair 0 slot 2) is never transformed: its contraction outputs are zero
// whatever its inputs, and k_bx reads that column of U1 as zero.
#include "common.cuh"
#include "contract_wl.cuh"
#include "fft4.cuh"
#include "ie_internal.h"
#include "tma.cuh"

namespace {

constexpr int kQB = 4;            // kx pairs per batch
constexpr int kChunk = 2;         // units per grab of a producer
constexpr int kStateHead = 4;     // next_unit, next_task, two spare
constexpr uint64_t kWaitNs = 2000000000ull;

template <typename R, int L, int NZ, int NP, int SL, int NG, int NSTAGE, bool PK, int NFW, int NL>
struct CfgY {
    static constexpr int P = NZ * (NZ + 1) / 2;
    static constexpr int T = 4 * P + 2 * NZ * NZ;
    static constexpr int ZL = NP * 3 * NZ;                 // lines of all vectors
    static constexpr int PTS = 4 * NP;
    static constexpr int ZW = 32 / SL;
    static constexpr int W = NZ / ZW;                      // warps per consumer group
    static constexpr int NC = NG * W * 32;                 // consumer threads
    static constexpr int NF = NFW * 32;                    // FFT threads
    static constexpr int NTHREADS = NC + 32 + NF;
    static constexpr int NR = 2 * 3 * PTS;
    static constexpr int ES = 2 * sizeof(R);
    static constexpr int TBYTES = T * ES;
    static constexpr int UBYTES = 4 * ZL * ES;
    static constexpr int STAGE_BYTES = TBYTES + UBYTES;
    static constexpr int N1 = Fact<L>::N1, N2 = Fact<L>::N2;
    static constexpr int LG_NL = Log2<NL>::v;
    static constexpr int NBLK = (ZL + NL - 1) / NL;        // line blocks per column
    static constexpr int IPT = (NL * N1 + NF - 1) / NF;    // step-1 items per FFT thread
    static constexpr int FFT_ELEMS = L + NL * (L + 1);     // twiddles + lines
    static constexpr int OFF_FFT = NSTAGE * STAGE_BYTES;
    static constexpr int OFF_BAR = OFF_FFT + FFT_ELEMS * ES;
    static constexpr int SMEM = OFF_BAR + 2 * NSTAGE * 8 + NSTAGE * 4 + 16;
    static_assert((1 << LG_NL) == NL, "lines per transform task must be a power of two");
    static_assert(NZ % ZW == 0 && 32 % SL == 0, "slices must tile a warp and warps the rows");
    static_assert(STAGE_BYTES % 16 == 0 && TBYTES % 16 == 0 && OFF_BAR % 8 == 0, "alignment");
    static_assert(SMEM <= 232448, "exceeds the 227 KB dynamic shared memory of one CTA");
    static_assert(NTHREADS <= 1024, "too many threads");
};

struct YArgs {
    const void *G;      // spectral tensor [q][r][T]
    void *Uh;           // spectrum [q][r][slot][ZL], in place
    void *U1;           // x-transformed vectors [kx][y][ZL]: forward input, inverse output
    const void *twy;    // y twiddles exp(-2 pi i j / 2Ny), j < 2Ny
    int *state;         // zeroed before the launch: grab counters, per-batch counts
    int *err;
    const int *gate;
    int Nx;
};

// Bounded wait until *p >= target (one thread); records `code` in *err on timeout and returns false.  Once
// any wait of the launch has given up (the error word is set) it returns at once, so the remaining tasks
// run through without adding 2 s each.
G2_D bool wait_count(const int *p, int target, int *err, int code)
{
    const volatile int *vp = p;
    if (*vp >= target) return true;
    const volatile int *ve = err;
    const uint64_t t0 = globaltimer_ns();
    while (*vp < target) {
        if (*ve != 0) return false;
        __nanosleep(128);
        if (globaltimer_ns() - t0 > kWaitNs) {
            atomicCAS(err, 0, code);
            return false;
        }
    }
    return true;
}

G2_D void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

template <typename C> G2_D C ld_l2(const C *p);
template <> G2_D double2 ld_l2<double2>(const double2 *p) { return __ldcg(p); }
template <> G2_D float2 ld_l2<float2>(const float2 *p) { return __ldcg(p); }

template <typename R, int L, int NZ, int NP, int SL, int NG, int NSTAGE, bool PK, int NFW, int NL>
__global__ void __launch_bounds__(CfgY<R, L, NZ, NP, SL, NG, NSTAGE, PK, NFW, NL>::NTHREADS, 1) k_ypipe(const YArgs a)
{
    if (a.gate && *a.gate == 0) return;  // uniform across the CTA: nothing has been issued yet
    using Cfg = CfgY<R, L, NZ, NP, SL, NG, NSTAGE, PK, NFW, NL>;
    using C2 = typename V2<R>::T;
    constexpr int ZL = Cfg::ZL, W = Cfg::W, Ny = L / 2;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *stages = smem;
    C2 *ftw = reinterpret_cast<C2 *>(smem + Cfg::OFF_FFT);  // y twiddles, then the transform lines
    C2 *fsm = ftw + L;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + Cfg::OFF_BAR);
    uint64_t *empty = full + NSTAGE;
    int *unit_of = reinterpret_cast<int *>(empty + NSTAGE);  // unit of each stage (-1: end of work)
    int *passed = unit_of + NSTAGE;                          // tickets [0, *passed) have been passed
    int *s_task = passed + 1;                                // FFT warps' current task

    const C2 *G = static_cast<const C2 *>(a.G);
    C2 *Uh = static_cast<C2 *>(a.Uh);
    C2 *U1 = static_cast<C2 *>(a.U1);
    int *err = a.err;
    const int Nx = a.Nx, nb = Nx / kQB;
    const int total_units = Nx * Ny;
    const int fpb = kQB * 2 * Cfg::NBLK;      // forward tasks per batch (inverse the same)
    const int cpb = kQB * Ny * W;              // warp arrivals per finished batch
    int *next_unit = a.state, *next_task = a.state + 1;
    int *f_done = a.state + kStateHead, *c_done = f_done + nb;

    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], W * 32);
        }
        *passed = 0;
        fence_mbar_init();
    }
    if (tid >= Cfg::NC + 32) {
        const C2 *twg = static_cast<const C2 *>(a.twy);
        for (int i = tid - (Cfg::NC + 32); i < L; i += Cfg::NF) ftw[i] = twg[i];
    }
    __syncthreads();

    if (tid >= Cfg::NC + 32) {
        // ------------------------------------ FFT warps ------------------------------------
        const int ftid = tid - (Cfg::NC + 32);
        auto fsync = [] { named_bar_sync(1, Cfg::NF); };
        const int n_tasks = 2 * nb * fpb;
        // the next task is grabbed while the current one runs (the atomic's round trip is hidden)
        if (ftid == 0) *s_task = atomicAdd(next_task, 1);
        fsync();
        while (true) {
            const int t = *s_task;
            fsync();
            int t_next = 0;
            if (ftid == 0 && t < n_tasks) t_next = atomicAdd(next_task, 1);
            if (t >= n_tasks) break;
            // segments: F(0), F(1), I(0), F(2), I(1), ..., F(nb-1), I(nb-2), I(nb-1)
            const int seg = t / fpb, within = t - seg * fpb;
            bool fwd;
            int b;
            if (seg == 0) { fwd = true; b = 0; }
            else if (seg == 2 * nb - 1) { fwd = false; b = nb - 1; }
            else if (seg & 1) { fwd = true; b = (seg + 1) / 2; }
            else { fwd = false; b = seg / 2 - 1; }
            const int qi = within / (2 * Cfg::NBLK), rem = within - qi * 2 * Cfg::NBLK;
            const int sx = rem / Cfg::NBLK, lb = rem - sx * Cfg::NBLK;
            const int q = b * kQB + qi, zl0 = lb * NL, nl = min(NL, ZL - zl0);
            if (!fwd) {
                if (ftid == 0) wait_count(&c_done[b], cpb, err, 43);
                fsync();
                __threadfence();
            }
            if (!(q == 0 && sx == 1)) {
                const int kx = sx ? 2 * Nx - q : q;
                C2 *col = U1 + (size_t)kx * Ny * ZL + zl0;
                C2 *spec = Uh + (size_t)q * Ny * 4 * ZL + sx * 2 * ZL + zl0;
                auto off = [&](int t2, int n1, int k2) { return t2 + NL * (n1 + Cfg::N1 * k2); };
                if (fwd) {
                    auto load = [&](int t2, int yy) -> C2 { return col[yy * ZL + t2]; };
                    auto store = [&](int t2, int ky, C2 v) {
                        int r, sy;
                        if (ky < Ny) { r = ky; sy = 0; }
                        else if (ky == Ny) { r = 0; sy = 1; }
                        else { r = 2 * Ny - ky; sy = 1; }
                        spec[(r * 4 + sy) * ZL + t2] = v;
                    };
                    fft4step_part_ilp<C2, Cfg::N1, Cfg::N2, Cfg::IPT, false, true, false>(
                        fsm, nl, Cfg::LG_NL, ftw, load, store, off, ftid, Cfg::NF, fsync);
                } else {
                    auto load = [&](int t2, int ky) -> C2 {
                        int r, sy;
                        if (ky < Ny) { r = ky; sy = 0; }
                        else if (ky == Ny) { r = 0; sy = 1; }
                        else { r = 2 * Ny - ky; sy = 1; }
                        return ld_l2(&spec[(r * 4 + sy) * ZL + t2]);
                    };
                    auto store = [&](int t2, int yy, C2 v) { col[yy * ZL + t2] = v; };
                    fft4step_part_ilp<C2, Cfg::N1, Cfg::N2, Cfg::IPT, true, false, true>(
                        fsm, nl, Cfg::LG_NL, ftw, load, store, off, ftid, Cfg::NF, fsync);
                }
            }
            if (fwd) __threadfence();
            fsync();  // every thread is done with the task (and its shared lines) before the next one
            if (ftid == 0) {
                if (fwd) atomicAdd(&f_done[b], 1);
                *s_task = t_next;
            }
            fsync();
        }
        return;
    }

    if (tid >= Cfg::NC) {
        // ------------------------------------ producer ------------------------------------
        if (tid != Cfg::NC) return;
        const uint64_t pol_t = l2_policy_evict_first();
        const uint64_t pol_u = l2_policy_evict_normal();
        int it = 0, ready_b = -1;
        bool ok = true;
        // units are grabbed kChunk at a time, and the next chunk is grabbed while this one is issued, so the
        // atomic's round trip stays out of the stage-refill path
        int u = atomicAdd(next_unit, kChunk), u_end = u + kChunk;
        int u_next = atomicAdd(next_unit, kChunk);
        while (true) {
            if (u >= u_end) {
                u = u_next;
                u_end = u + kChunk;
                if (u < total_units) u_next = atomicAdd(next_unit, kChunk);
            }
            if (u >= total_units) break;
            const int slot = it % NSTAGE;
            const uint32_t round = (uint32_t)(it / NSTAGE);
            if (round > 0 && !mbar_wait_bounded(&empty[slot], (round - 1) & 1, err, 41)) { ok = false; break; }
            unsigned char *st = stages + slot * Cfg::STAGE_BYTES;
            unit_of[slot] = u;
            mbar_arrive_expect_tx(&full[slot], Cfg::STAGE_BYTES);
            bulk_g2s(st, G + (size_t)u * Cfg::T, Cfg::TBYTES, &full[slot], pol_t);
            const int b = (u / Ny) / kQB;
            if (b > ready_b) {
                wait_count(&f_done[b], fpb, err, 42);  // on timeout: go on, the error word is set
                __threadfence();
                fence_proxy_async_global();
                ready_b = b;
            }
            bulk_g2s(st + Cfg::TBYTES, Uh + (size_t)u * 4 * ZL, Cfg::UBYTES, &full[slot], pol_u);
            it++;
            u++;
        }
        if (ok) {
            // one end-of-work ticket per consumer group
            for (int k = 0; k < NG; k++, it++) {
                const int slot = it % NSTAGE;
                const uint32_t round = (uint32_t)(it / NSTAGE);
                if (round > 0 && !mbar_wait_bounded(&empty[slot], (round - 1) & 1, err, 41)) break;
                unit_of[slot] = -1;
                mbar_arrive(&full[slot]);
            }
        } else {
            // the consumers stopped: every copy in flight must land before the CTA may exit
            for (int k = (it > NSTAGE ? it - NSTAGE : 0); k < it; k++)
                mbar_wait_bounded(&full[k % NSTAGE], (uint32_t)(k / NSTAGE) & 1, err, 46);
        }
        return;
    }

    // ------------------------------------ consumers ------------------------------------
    const int warp = tid >> 5, lane = tid & 31;
    const int g = warp / W, z = (warp % W) * Cfg::ZW + lane % Cfg::ZW, s = lane / Cfg::ZW;
    for (int it = g;; it += NG) {
        const int slot = it % NSTAGE;
        const uint32_t round = (uint32_t)(it / NSTAGE);
        if (!__all_sync(0xffffffffu, wait_ticket(passed, it, err, 44))) return;
        __threadfence_block();
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&full[slot], round & 1, err, 45))) return;
        __threadfence_block();
        if (lane == 0) atomicMax(passed, it + 1);
        const int u = *reinterpret_cast<volatile int *>(&unit_of[slot]);
        if (u < 0) {
            // end of work for this group; the stage goes back too, since with more groups than stages the
            // producer puts later end tickets into it
            mbar_arrive(&empty[slot]);
            return;
        }
        const unsigned char *st = stages + slot * Cfg::STAGE_BYTES;
        R v[Cfg::NR];
        wl_unit_sums<R, NZ, SL, NP, false, PK>(reinterpret_cast<const C2 *>(st),
                                                reinterpret_cast<const C2 *>(st + Cfg::TBYTES), z, s, v);
        mbar_arrive(&empty[slot]);  // this lane's reads of the stage are done
        const int q = u / Ny, r = u - q * Ny;
        wl_unit_store<R, NZ, SL, NP>(v, s, q, r, Uh + (size_t)u * 4 * ZL + z);
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicAdd(&c_done[q / kQB], 1);
    }
}

int sm_count_y()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    }
    return n;
}

template <typename R, int L, int NZ, int NP, int SL, int NG, int NSTAGE, bool PK, int NFW, int NL>
int launch_y(const YArgs &a, size_t state_bytes, cudaStream_t st)
{
    using Cfg = CfgY<R, L, NZ, NP, SL, NG, NSTAGE, PK, NFW, NL>;
    auto kern = k_ypipe<R, L, NZ, NP, SL, NG, NSTAGE, PK, NFW, NL>;
    static bool attr = false;
    if (!attr) {
        G2_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM));
        attr = true;
    }
    G2_CUDA_CHECK(cudaMemsetAsync(a.state, 0, state_bytes, st));
    kern<<<sm_count_y(), Cfg::NTHREADS, Cfg::SMEM, st>>>(a);
    G2_CUDA_CHECK(cudaGetLastError());
    return G2_OK;
}

// variant: the tile shapes of the three forms (precision 0, 1, 2 = paired complex64).  Block sizes are
// multiples of 128 threads (registers are allotted per four warps): FP64 2 groups of 4 consumer warps +
// producer + 3 FFT warps = 384; complex64 4 or 6 groups of 2 warps + 1 + 3 = 384 or 512.  The slices per
// row (SL) and the packed complex64 form match the stand-alone contraction's tuned shapes (k_contract_wl
// FP64 SL = 4, complex64 SL = 2 packed), so both paths sum in the same order.
template <int L>
int dispatch_nz32(int prec, int variant, const YArgs &a, size_t sb, cudaStream_t st)
{
    constexpr int NLW = L >= 512 ? 8 : 16;  // lines per transform task (the 2Ny = 512 tile is twice as long)
    if (prec == 0) {
        if (variant == 1) return launch_y<double, L, 32, 1, 4, 2, 2, false, 3, 8>(a, sb, st);
        return launch_y<double, L, 32, 1, 4, 2, 2, false, 3, NLW>(a, sb, st);
    }
    if (prec == 1) {
        if (variant == 1) return launch_y<float, L, 32, 1, 2, 4, 5, true, 3, NLW>(a, sb, st);
        return launch_y<float, L, 32, 1, 2, 6, 5, true, 3, NLW>(a, sb, st);
    }
    if (variant == 1) return launch_y<float, L, 32, 2, 2, 4, 4, true, 3, 8>(a, sb, st);
    return launch_y<float, L, 32, 2, 2, 4, 4, true, 3, NLW>(a, sb, st);
}

}  // namespace

// The pipelined y-pass exists for Nz = 32, 2Ny in {64, 128, 256, 512} and Nx a multiple of the batch (4).
bool ie_ypipe_supported(int Nx, int Ny, int Nz)
{
    return Nz == 32 && (Ny == 32 || Ny == 64 || Ny == 128 || Ny == 256) && Nx % kQB == 0 && Nx >= kQB;
}
int ie_ypipe_variants(int precision) { (void)precision; return 2; }
size_t ie_ypipe_state_bytes(int Nx) { return (size_t)(kStateHead + 2 * (Nx / kQB)) * sizeof(int); }

// U1 -> (forward y-FFT, contraction, inverse y-FFT) -> U1, the spectrum Uh as in-place scratch.
// precision 0: complex128 (double2 buffers); 1: complex64; 2: two complex64 vectors sharing the tensor.
int ie_ypipe(IeOp *op, int precision, const void *G, void *U1, void *Uh, int *state, cudaStream_t st,
             const int *gate)
{
    if (!ie_ypipe_supported(op->Nx, op->Ny, op->Nz)) return G2_ERR_UNSUPPORTED;
    YArgs a;
    a.G = G;
    a.Uh = Uh;
    a.U1 = U1;
    a.twy = precision == 0 ? static_cast<const void *>(op->d_twy64) : static_cast<const void *>(op->d_twy32);
    a.state = state;
    a.err = op->d_err;
    a.gate = gate;
    a.Nx = op->Nx;
    const size_t sb = ie_ypipe_state_bytes(op->Nx);
    const int v = op->ypipe_mode[precision < 0 || precision > 2 ? 0 : precision];
    switch (op->Ny) {
    case 32: return dispatch_nz32<64>(precision, v, a, sb, st);
    case 64: return dispatch_nz32<128>(precision, v, a, sb, st);
    case 128: return dispatch_nz32<256>(precision, v, a, sb, st);
    case 256: return dispatch_nz32<512>(precision, v, a, sb, st);
    default: return G2_ERR_UNSUPPORTED;
    }
}
