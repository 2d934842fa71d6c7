// Pieces shared by the two Hankel-transform tensor builders on the GPU: the IE Green's tensor
// (green.cu, calc_ie_tensor_module.F90) and the receiver tensor (continuation.cu,
// calc_rc_tensor_module.F90).
//   * the volume Bessel transform tables (VolumeBesselTransforms.F90:111-139) and the FFT deconvolution
//     that turns 1024 samples of an output function into the 501 Hankel weights (CalcWeights22,
//     :264-288);
//   * the layered-medium recursions of apq_module.F90 (Calc_Apq, Calc_p, Calc_q, Calc_pexpz_All,
//     Calc_qexpz_All) for one lambda, on one thread, 1-based layer and cell arrays;
//   * the FP64 GEMM that sums weights x lambda basis into the tensor.
// Everything sits in an anonymous namespace: each translation unit gets its own copy.
#pragma once
#include <cmath>
#include <vector>
#include <cuda/std/complex>
#include "common.cuh"

namespace {

using cplx = cuda::std::complex<double>;

constexpr int VN = 1024, VLOG = 10, NFIRST = 212, NLAST = 712, NLAM = NLAST - NFIRST + 1;
constexpr double Y_STEP = 1e-1 * 2e0;
constexpr double XI = -4.82205425726955430357775925664462079e-2 * 2e0;
constexpr double VQ = Y_STEP / 2.0;
constexpr double VP = VQ + XI;
constexpr int VN2 = -VN / 2;
constexpr double PI_D = 3.14159265358979323846264338327950288;
constexpr double SPI = 1.77245385090551602729816748334114518;
constexpr double WT_THRESHOLD = 1e-12;
constexpr int MAXL = 16;   // layers supported by the device recursion
constexpr int MAXZ = 64;   // cells in z supported by the device recursion

struct Bkg {
    int Nl, Nz;
    double2 csigma[MAXL + 1];  // 0..Nl
    double2 k2[MAXL + 1];
    double thick[MAXL + 1];    // 1..Nl-1
    double depth[MAXL + 1];    // 1..Nl-1
    double2 iwm;
    int L[MAXZ + 1];           // Lnumber 0..Nz
    double z[MAXZ + 1];        // 0..Nz
    double dz[MAXZ + 1];       // 1..Nz
};

G2_D cplx C(double2 v) { return cplx(v.x, v.y); }
G2_D double2 D2(cplx v) { return make_double2(v.real(), v.imag()); }

// Calc_Apq without the A matrix (apq_module.F90:230-248) with Calc_p (:267-290) and Calc_q (:291-312)
G2_D void dev_apq(const Bkg &b, double lms, cplx *eta, cplx *el, cplx (*p)[2], cplx (*q)[2], cplx (*Arr)[2])
{
    const int Nl = b.Nl;
    const cplx cs0 = C(b.csigma[0]);
    for (int i = 1; i <= Nl; i++) eta[i] = cuda::std::sqrt(lms * lms - C(b.k2[i]));
    for (int i = 1; i <= Nl - 1; i++) el[i] = cuda::std::exp(-2.0 * eta[i] * b.thick[i]);
    el[Nl] = 0.0;
    {  // Calc_p (:267-290)
        const cplx eta0 = cuda::std::sqrt(lms * lms - C(b.k2[0]));
        const cplx ceta = eta0 / eta[1];
        p[1][0] = (1.0 - ceta) / (1.0 + ceta);
        const cplx cgamma = cs0 / C(b.csigma[1]);
        p[1][1] = (cgamma - ceta) / (cgamma + ceta);
        for (int i = 2; i <= Nl; i++) {
            cplx w[2] = {el[i - 1] * p[i - 1][0], el[i - 1] * p[i - 1][1]};
            for (int k = 0; k < 2; k++) w[k] = (w[k] - 1.0) / (w[k] + 1.0);
            cplx a[2];
            a[0] = eta[i - 1] / eta[i];
            a[1] = a[0] * C(b.csigma[i]) / C(b.csigma[i - 1]);
            for (int k = 0; k < 2; k++) {
                w[k] = w[k] * a[k];
                p[i][k] = (1.0 + w[k]) / (1.0 - w[k]);
            }
        }
    }
    {  // Calc_q (:291-312)
        q[Nl][0] = q[Nl][1] = 0.0;
        if (Nl > 1) {
            cplx a[2];
            a[0] = eta[Nl] / eta[Nl - 1];
            a[1] = a[0] * C(b.csigma[Nl - 1]) / C(b.csigma[Nl]);
            for (int k = 0; k < 2; k++) q[Nl - 1][k] = (1.0 - a[k]) / (1.0 + a[k]);
            for (int i = Nl - 2; i >= 1; i--) {
                cplx w[2] = {el[i + 1] * q[i + 1][0], el[i + 1] * q[i + 1][1]};
                for (int k = 0; k < 2; k++) w[k] = (w[k] - 1.0) / (w[k] + 1.0);
                a[0] = eta[i + 1] / eta[i];
                a[1] = a[0] * C(b.csigma[i]) / C(b.csigma[i + 1]);
                for (int k = 0; k < 2; k++) {
                    w[k] = w[k] * a[k];
                    q[i][k] = (1.0 + w[k]) / (1.0 - w[k]);
                }
            }
        }
    }
    for (int i = 1; i <= Nl; i++)
        for (int k = 0; k < 2; k++) Arr[i][k] = 1.0 / eta[i] / (1.0 - p[i][k] * q[i][k] * el[i]);
}

// Calc_pexpz_All (apq_module.F90:112-137): pez[i] for cells 1..Nz
G2_D void dev_pexpz(const Bkg &b, const cplx *eta, const cplx (*p)[2], const cplx *expz, cplx (*pez)[2])
{
    const int Nz = b.Nz;
    int l = b.L[0];
    cplx e;
    if (l > 1) e = cuda::std::exp(-2.0 * eta[l] * (b.z[0] - b.depth[l - 1]));
    else if (l == 1) e = cuda::std::exp(-2.0 * eta[1] * b.z[0]);
    else e = 1.0;
    for (int i = 1; i <= Nz; i++) {
        if (l != b.L[i]) e = 1.0;
        l = b.L[i];
        pez[i][0] = e * p[l][0];
        pez[i][1] = e * p[l][1];
        e = e * expz[i] * expz[i];
    }
}

// Calc_qexpz_All (apq_module.F90:155-177): qez[i] for cells 1..Nz
G2_D void dev_qexpz(const Bkg &b, const cplx *eta, const cplx (*q)[2], const cplx *expz, cplx (*qez)[2])
{
    const int Nz = b.Nz, Nl = b.Nl;
    int l = b.L[Nz];
    cplx e;
    if (l != Nl) e = cuda::std::exp(-2.0 * eta[l] * (b.depth[l] - b.z[Nz]));
    else e = 0.0;
    for (int i = Nz; i >= 1; i--) {
        if (l != b.L[i]) e = 1.0;
        l = b.L[i];
        qez[i][0] = e * q[l][0];
        qez[i][1] = e * q[l][1];
        e = e * expz[i] * expz[i];
    }
}

struct VbtTab {
    int inds[VN];
    double2 twf[VN / 2];  // exp(-i pi j / (VN/2)) style table for smem_fft: exp(-2 pi i j / VN), j < VN/2
    double2 f1[VN];
    double lms[NLAM];
    double lambda_shift;
};

// CalcWeights22 (VolumeBesselTransforms.F90:264-288) after the output function's samples are in g
// ([VN][6] in shared memory, bit-reversed positions): forward FFT, deconvolution by the input function's
// spectrum, inverse FFT.  The caller normalises (h/N with the alternating sign) and takes the real part.
// Needs blockDim.x == 256 and a __syncthreads() between filling g and the call.
G2_D void vbt_weights22(double2 *g, const VbtTab *__restrict__ T)
{
    smem_fft<double2, true>(g, VLOG, 6, 1, 6, T->twf, false);
    // deconvolution by the input function's spectrum, written back bit-reversed (CalcWeights22 :277-280);
    // every thread reads its pairs before any thread writes (the permutation is in place)
    static_assert(VN / 2 == 2 * 256, "k_weights is written for 256 threads, two sample pairs each");
    double2 pa[2][6], pb[2][6];
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int j = 2 * (threadIdx.x + r * 256);
#pragma unroll
        for (int c = 0; c < 6; c++) { pa[r][c] = g[j * 6 + c]; pb[r][c] = g[(j + 1) * 6 + c]; }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int j = 2 * (threadIdx.x + r * 256);
        const cplx f0 = C(T->f1[j]), f1v = C(T->f1[j + 1]);
        const int p0 = T->inds[j], p1 = T->inds[j + 1];
#pragma unroll
        for (int c = 0; c < 6; c++) {
            g[p0 * 6 + c] = D2(C(pa[r][c]) / f0);
            g[p1 * 6 + c] = D2(-C(pb[r][c]) / f1v);
        }
    }
    __syncthreads();
    smem_fft<double2, true>(g, VLOG, 6, 1, 6, T->twf, true);
}

// ---- (3) GEMM: out[lag][off + col] = scale * sum_k (A1[lag][k] B1[k][col] + A2[lag][k] B2[k][col]) --------
constexpr int GM = 32, GN = 32, GK = 16;
__global__ void __launch_bounds__(256) k_gemm(const double *__restrict__ A1, const double2 *__restrict__ B1,
                                              const double *__restrict__ A2, const double2 *__restrict__ B2,
                                              int nlags, int ncols, double2 *out, int T, int off, double scale)
{
    __shared__ double As[2][GK][GM + 1];
    __shared__ double2 Bs[2][GK][GN];
    const int m0 = blockIdx.x * GM, n0 = blockIdx.y * GN;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads, 2 x 2 outputs each
    double2 acc[2][2] = {};
    const int npair = A2 ? 2 : 1;
    for (int pr = 0; pr < npair; pr++) {
        const double *A = pr ? A2 : A1;
        const double2 *B = pr ? B2 : B1;
        for (int k0 = 0; k0 < NLAM; k0 += GK) {
            for (int i = threadIdx.x; i < GM * GK; i += 256) {
                const int mm = i / GK, kk = i - mm * GK;
                const int gm = m0 + mm, gk = k0 + kk;
                As[pr][kk][mm] = (gm < nlags && gk < NLAM) ? A[(size_t)gm * NLAM + gk] : 0.0;
            }
            for (int i = threadIdx.x; i < GK * GN; i += 256) {
                const int kk = i / GN, nn = i - kk * GN;
                const int gk = k0 + kk, gn = n0 + nn;
                Bs[pr][kk][nn] = (gk < NLAM && gn < ncols) ? B[(size_t)gk * ncols + gn] : make_double2(0.0, 0.0);
            }
            __syncthreads();
#pragma unroll
            for (int kk = 0; kk < GK; kk++) {
                const double a0 = As[pr][kk][ty * 2], a1 = As[pr][kk][ty * 2 + 1];
                const double2 b0 = Bs[pr][kk][tx * 2], b1 = Bs[pr][kk][tx * 2 + 1];
                acc[0][0].x = fma(a0, b0.x, acc[0][0].x); acc[0][0].y = fma(a0, b0.y, acc[0][0].y);
                acc[0][1].x = fma(a0, b1.x, acc[0][1].x); acc[0][1].y = fma(a0, b1.y, acc[0][1].y);
                acc[1][0].x = fma(a1, b0.x, acc[1][0].x); acc[1][0].y = fma(a1, b0.y, acc[1][0].y);
                acc[1][1].x = fma(a1, b1.x, acc[1][1].x); acc[1][1].y = fma(a1, b1.y, acc[1][1].y);
            }
            __syncthreads();
        }
    }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            const int gm = m0 + ty * 2 + i, gn = n0 + tx * 2 + j;
            if (gm < nlags && gn < ncols)
                out[(size_t)gm * T + off + gn] = make_double2(acc[i][j].x * scale, acc[i][j].y * scale);
        }
}

// ---- host tables (VolumeBesselTransforms.F90:111-139) -------------------------------------------
int bitrev_vbt(int i)
{
    int t = i;
    for (int J = VLOG; J >= 2; J--) {
        const int mask = (1 << J) - 1;
        int low = t & mask;
        low = (low >> 1) | ((low & 1) << (J - 1));
        t = (t & ~mask) | low;
    }
    return t;
}
double input_function(double t)
{
    const double y = std::exp(-t), y2 = y * y, y4 = y2 * y2;
    return 8.0 * std::exp(-y2) * (y4 - 4.0 * y2 + 2.0) * y;
}
void make_vbt(double s, VbtTab &T)
{
    for (int i = 0; i < VN; i++) T.inds[i] = bitrev_vbt(i);
    for (int j = 0; j < VN / 2; j++) {
        const double th = -2.0 * PI_D * j / VN;
        T.twf[j] = make_double2(std::cos(th), std::sin(th));
    }
    for (int J = NFIRST; J <= NLAST; J++) T.lms[J - NFIRST] = std::exp(XI + (J + VN2) * Y_STEP) / s;
    T.lambda_shift = std::log(s);
    std::vector<double2> f(VN);
    for (int i = 0; i < VN; i += 2) {
        double y1 = (i + VN2) * Y_STEP + VQ;
        f[T.inds[i]] = make_double2(input_function(y1), 0.0);
        y1 = y1 + Y_STEP;
        f[T.inds[i + 1]] = make_double2(-input_function(y1), 0.0);
    }
    // radix-2 DIT on bit-reversed input (FFT_16, :630-649)
    for (int h = 1; h < VN; h <<= 1)
        for (int J = 0; J < h; J++) {
            const double th = -PI_D / h * J;
            const double wr = std::cos(th), wi = std::sin(th);
            for (int ip = J; ip < VN; ip += 2 * h) {
                const int iq = ip + h;
                const double tr = wr * f[iq].x - wi * f[iq].y, ti = wr * f[iq].y + wi * f[iq].x;
                f[iq] = make_double2(f[ip].x - tr, f[ip].y - ti);
                f[ip] = make_double2(f[ip].x + tr, f[ip].y + ti);
            }
        }
    for (int i = 0; i < VN; i++) T.f1[i] = f[i];
}

}  // namespace
