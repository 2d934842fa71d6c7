// Receiver continuation on the GPU, FP64: electric and magnetic fields at receiver points from the
// currents j = (csiga - csigb) E of an IE solution.
//
// Restates Continuation_Function_Module.F90 (RC_OPERATOR, CalcFFTofRCTensor :330-366, ReCalculation
// :198-239, LoadEint :240-263, APPLY_RC_E_OP / APPLY_RC_H_OP :382-481), calc_rc_tensor_module.F90
// (CalcRecalculationGreenTensor :38-229) and rc_kernel_hankel_module.F90 (Calc_Integral_U :56-145,
// Calc_G_not_match :147-179, Calc_Recv_Part :181-225, Calc_Ftb :227-252).
//
// Tensor.  For receiver r, lateral lag (lx, ly) and source cell z the reference sums, over the lambdas
// whose single-integral Hankel weights pass the 1e-12 threshold, products of the six weights
// WT(lambda; lag, r) with eight lambda functions G(lambda; z, r) (Calc_G_not_match).  The G functions do
// not depend on the lag, and the sums are linear in the weights, so the GPU computes
//   (1) k_rc_basis:   per (lambda, receiver): the 13 products the 15 components need, over z;
//   (2) k_rc_weights: per (lag, receiver): the 501 x 6 weights (1024-point FFT deconvolution), the
//                     threshold mask and the lambda scalings;
//   (3) k_gemm:       component(lag; r, z) = sum_lambda sum_w W_w(lag, lambda) B_{c,w}(lambda; r, z) / (4 pi).
// A lambda that the reference skips for a lag has all six weights zero here, so the sums hold the same
// terms; only the order of the floating-point additions differs.  The tensor covers the whole
// 2Nx x 2Ny lag plane (index ix < Nx is lag ix, ix > Nx is lag ix - 2Nx, ix = Nx is zero; same in y),
// layout [2Ny][2Nx][15][Nr][Nz] with components E: xx xy xz yy yz zx zy zz, H: xx xy xz yx yz zx zy
// (const_module.F90:112-130).  It is transformed to its unnormalised 2-D spectrum in place.
//
// Apply.  The reference transforms the currents twice (once for E, once for H) and runs nine and eight
// ZGEMVs per spectral point.  Here one forward transform feeds one contraction that produces all six
// field components, and one inverse transform of 6 Nr components gives Ea and Ha:
//   k_rc_pass<CURRENTS>  x-FFT of dsig * E for rows y < Ny (the zero padding is not loaded)
//   k_rc_pass<GENERIC>   y-FFT (rows >= Ny are zero and not loaded)
//   k_rc_contract        per spectral point: Ea_c(r) += sum_z G(c, r, z) j(z)  (warp per point, lanes on z)
//   k_rc_pass<GENERIC>   inverse y-FFT, rows y < Ny kept
//   k_rc_pass<FIELDS>    inverse x-FFT, x < Nx kept, divided by 4 Nx Ny (RC_OP_FFTW_BWD :324-328)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "common.cuh"
#include "ie_internal.h"
#include "rc_internal.h"
#include "hankel.cuh"

namespace {

constexpr int RC_NCOMP = 15;  // 8 E slots, 7 H slots
constexpr int RC_NBASIS = 13;
enum { RC_DXX = 0, RC_DXY = 1, RC_DYY = 2, RC_DX = 3, RC_DY = 4, RC_D0 = 5 };  // rc_kernel_hankel_module.F90:31-38
enum { REXX = 0, REXY, REXZ, REYY, REYZ, REZX, REZY, REZZ, RHXX, RHXY, RHXZ, RHYX, RHYZ, RHZX, RHZY };
// basis products: G11 = G1 iwm, G3DZ + G11, G2DZ, G2DZ0, G2G2DZZ, G3, -G1DZ, G2, G1DZ, -G3, -G2, -G1, G1
enum { B_G11 = 0, B_G3DZ_G11, B_G2DZ, B_G2DZ0, B_G2G2DZZ, B_G3, B_MG1DZ, B_G2, B_G1DZ, B_MG3, B_MG2, B_MG1, B_G1 };

struct RcRecvDev {
    double zrecv;
    int layer, anom_cell;
};

// ---- (1) lambda basis -----------------------------------------------------------------------------
// B layout: [Nr][13][NLAM][Nz]
__global__ void __launch_bounds__(64) k_rc_basis(const Bkg *__restrict__ bk, const RcRecvDev *__restrict__ recv,
                                                 const double *__restrict__ lms_all, double2 *B)
{
    const int li = blockIdx.x, r = blockIdx.y;
    const double lms = lms_all[li];
    const Bkg &b = *bk;
    const int Nl = b.Nl, Nz = b.Nz;
    const RcRecvDev rv = recv[r];
    const int rl = rv.layer;
    __shared__ cplx s_eta[MAXL + 1], s_p[MAXL + 1][2], s_q[MAXL + 1][2], s_A[MAXL + 1][2];
    __shared__ cplx s_expz[MAXZ + 1], s_pez[MAXZ + 1][2], s_qez[MAXZ + 1][2];
    if (threadIdx.x == 0) {
        cplx eta[MAXL + 1], el[MAXL + 1], p[MAXL + 1][2], q[MAXL + 1][2], Arr[MAXL + 1][2];
        dev_apq(b, lms, eta, el, p, q, Arr);
        // row rl of the layer-transfer matrix A of Calc_Apq (apq_module.F90:249-264):
        //   A(J,I) = A(J+1,I) w(J) for J < I, A(I,I) = Arr(I), A(I,J,1) = A(J,I,1),
        //   A(I,J,2) = A(J,I,2) csigma(I) / csigma(J)
        cplx w[MAXL + 1][2];
        for (int i = 1; i <= Nl - 1; i++) {
            cplx tmp = C(b.k2[i]) - C(b.k2[i + 1]);
            tmp = b.depth[i] * tmp;
            tmp = tmp / (eta[i + 1] + eta[i]);
            for (int k = 0; k < 2; k++) w[i][k] = (1.0 + p[i + 1][k]) / (1.0 + p[i][k] * el[i]) * cuda::std::exp(tmp);
        }
        for (int l = 1; l <= Nl; l++) {
            if (l >= rl) {  // A(rl, l) = A(rl+1, l) w(rl) ... from A(l, l) = Arr(l)
                cplx a0 = Arr[l][0], a1 = Arr[l][1];
                for (int j = l - 1; j >= rl; j--) {
                    a0 = a0 * w[j][0];
                    a1 = a1 * w[j][1];
                }
                s_A[l][0] = a0;
                s_A[l][1] = a1;
            } else {        // A(rl, l) from A(l, rl)
                cplx a0 = Arr[rl][0], a1 = Arr[rl][1];
                for (int j = rl - 1; j >= l; j--) {
                    a0 = a0 * w[j][0];
                    a1 = a1 * w[j][1];
                }
                s_A[l][0] = a0;
                s_A[l][1] = a1 * C(b.csigma[rl]) / C(b.csigma[l]);
            }
        }
        // expz (rc_kernel_hankel_module.F90:84-87), pexpz / qexpz (apq_module.F90:112-177)
        cplx expz[MAXZ + 1], pez[MAXZ + 1][2], qez[MAXZ + 1][2];
        for (int iz = 1; iz <= Nz; iz++) expz[iz] = cuda::std::exp(-eta[b.L[iz]] * (b.z[iz] - b.z[iz - 1]));
        dev_pexpz(b, eta, p, expz, pez);
        dev_qexpz(b, eta, q, expz, qez);
        for (int i = 1; i <= Nl; i++) {
            s_eta[i] = eta[i];
            for (int k = 0; k < 2; k++) {
                s_p[i][k] = p[i][k];
                s_q[i][k] = q[i][k];
            }
        }
        for (int iz = 1; iz <= Nz; iz++) {
            s_expz[iz] = expz[iz];
            for (int k = 0; k < 2; k++) {
                s_pez[iz][k] = pez[iz][k];
                s_qez[iz][k] = qez[iz][k];
            }
        }
    }
    __syncthreads();
    const double lm2 = lms * lms;
    const cplx iwm = C(b.iwm), csr = C(b.csigma[rl]);
    const cplx eta_r = s_eta[rl];
    const cplx eta_zr = eta_r * rv.zrecv;
    const int N = rv.anom_cell;
    for (int iz = threadIdx.x + 1; iz <= Nz; iz += blockDim.x) {
        const int l = b.L[iz];
        // Calc_Recv_Part (:181-225)
        cplx w1[2], w2[2];
        if (iz >= N + 1) {  // cell below the receiver
            const cplx eta_dr = rl > 1 ? eta_r * b.depth[rl - 1] * 2.0 : cplx(0.0);
            const cplx e1 = cuda::std::exp(-b.z[iz - 1] * s_eta[l] + eta_zr);
            const cplx e2 = cuda::std::exp(-b.z[iz - 1] * s_eta[l] - eta_zr + eta_dr);
            w1[0] = (e2 * s_p[rl][0] + e1);
            w1[1] = (-e2 * s_p[rl][0] + e1) * eta_r;
            w2[0] = (e2 * s_p[rl][1] + e1);
            w2[1] = (-e2 * s_p[rl][1] + e1) * eta_r;
        } else {            // cell above the receiver
            const cplx eta_dr = rl < Nl ? eta_r * b.depth[rl] * 2.0 : cplx(1.7976931348623157e308);  // HUGE
            const cplx e1 = cuda::std::exp(b.z[iz] * s_eta[l] - eta_zr);
            const cplx e2 = cuda::std::exp(b.z[iz] * s_eta[l] + eta_zr - eta_dr);
            w1[0] = (e2 * s_q[rl][0] + e1);
            w1[1] = (e2 * s_q[rl][0] - e1) * eta_r;
            w2[0] = (e2 * s_q[rl][1] + e1);
            w2[1] = (e2 * s_q[rl][1] - e1) * eta_r;
        }
        // Calc_Ftb (:227-252): cells above the receiver use pexpz with sign -1, cells below qexpz with +1
        const bool above = (N > Nz) || (N >= 1 && iz <= N);
        const cplx *pq = above ? s_pez[iz] : s_qez[iz];
        const double sg = above ? -1.0 : 1.0;
        const cplx ez = s_expz[iz];
        const cplx a = (1.0 - ez);
        const cplx a1 = a / s_eta[l];
        const cplx e10 = 1.0 + pq[0] * ez, e11 = 1.0 + pq[1] * ez;
        const cplx e21 = (1.0 - pq[1] * ez) * sg;
        const cplx f0 = a1 * e10, f1 = a1 * e11, f2 = a * e21;
        // Calc_G_not_match (:147-179)
        const cplx A1 = s_A[l][0], A2 = s_A[l][1];
        const cplx G1 = A1 * f0 * w1[0];
        const cplx G3DZ = (A2 * f2 * w2[1]) / csr;
        const cplx G2DZ = (A2 * f1 * w2[1]) / csr;
        const cplx G2DZ0 = (A2 * f2 * w2[0]) / csr;
        const cplx G2G2DZZ = lm2 * (A2 * f1 * w2[0]) / csr;
        const cplx G3 = (A2 * f2 * w2[0] - A1 * f0 * w1[1]);
        const cplx G1DZ = A1 * f0 * w1[1];
        const cplx G2 = A2 * f1 * w2[0];
        const cplx G11 = G1 * iwm;
        const cplx v[RC_NBASIS] = {G11, G3DZ + G11, G2DZ, G2DZ0, G2G2DZZ, G3, -G1DZ, G2, G1DZ, -G3, -G2, -G1, G1};
        double2 *out = B + ((size_t)r * RC_NBASIS * NLAM + li) * Nz + (iz - 1);
#pragma unroll
        for (int k = 0; k < RC_NBASIS; k++) out[(size_t)k * NLAM * Nz] = D2(v[k]);
    }
}

// ---- (2) single-integral weights per lag ----------------------------------------------------------
// SINGLE_INT_D0 / D1 / D2 (VolumeBesselTransforms.F90:553-603) on the two edges k = 0, 1
G2_D void sint_d0(const double *x, const double *x2, const double *ex, const double *er, double R[3])
{
    double f[2];
    for (int k = 0; k < 2; k++) f[k] = er[k] * SPI;
    const double a = f[1] - f[0];
    R[0] = a * 0.5;
    for (int k = 0; k < 2; k++) f[k] = x[k] * ex[k];
    const double b = f[1] - f[0];
    R[1] = a - 2.0 * b;
    for (int k = 0; k < 2; k++) f[k] = f[k] * x2[k];
    const double c = f[1] - f[0];
    R[2] = 6.0 * a - 12.0 * b - 8.0 * c;
}
G2_D void sint_d1(const double *x2, const double *ex, double R[3])
{
    double f[2];
    for (int k = 0; k < 2; k++) f[k] = ex[k];
    R[0] = f[1] - f[0];
    for (int k = 0; k < 2; k++) f[k] = f[k] * x2[k];
    R[1] = f[1] - f[0];
    for (int k = 0; k < 2; k++) f[k] = f[k] * x2[k];
    R[2] = f[1] - f[0];
    R[0] = R[0] / 2.0;
    R[1] = R[1] * 2.0;
    R[2] = R[2] * 8.0;
}
G2_D void sint_d2(const double *x, const double *x2, const double *ex, double R[3])
{
    double f[2];
    for (int k = 0; k < 2; k++) f[k] = x[k] * ex[k];
    const double a = f[1] - f[0];
    R[0] = -a * 0.5;
    for (int k = 0; k < 2; k++) f[k] = f[k] * x2[k];
    const double b = f[1] - f[0];
    R[1] = 2.0 * (a - b);
    for (int k = 0; k < 2; k++) f[k] = f[k] * x2[k];
    const double c = f[1] - f[0];
    R[2] = 16.0 * b - 8.0 * c;
}

// CALC_EXP_LT (:142-157), PrepareExps2 (:342-371) and outfunc_int2_all (:407-434) for sample i
G2_D void outfunc2(int i, double s_arg, double cphi, double sphi, double alpha, double beta, double R[6])
{
    const int i0 = i & ~1;
    double y2 = (i0 + VN2) * Y_STEP + VP + s_arg;
    if (i & 1) y2 = y2 + Y_STEP;
    const double ex1 = exp(y2);
    const double x1 = ex1 * cphi * 0.5, y1 = ex1 * sphi * 0.5;
    const double dxv = alpha * ex1 * 0.5, dyv = beta * ex1 * 0.5;
    double xv[2] = {x1, x1 + dxv}, yv[2] = {y1, y1 + dyv};
    double x2[2], y2v[2], xe[2], ye[2], xr[2], yr[2];
    for (int k = 0; k < 2; k++) {
        x2[k] = xv[k] * xv[k];
        xe[k] = exp(-x2[k]);
        xr[k] = erf(xv[k]);
        y2v[k] = yv[k] * yv[k];
        ye[k] = exp(-y2v[k]);
        yr[k] = erf(yv[k]);
    }
    double fx[3][3], fy[3][3];
    sint_d0(xv, x2, xe, xr, fx[0]);
    sint_d1(x2, xe, fx[1]);
    sint_d2(xv, x2, xe, fx[2]);
    sint_d0(yv, y2v, ye, yr, fy[0]);
    sint_d1(y2v, ye, fy[1]);
    sint_d2(yv, y2v, ye, fy[2]);
#define FX(k, D) fx[D][(k)-1]
#define FY(k, D) fy[D][(k)-1]
    R[0] = FX(3, 0) * FY(1, 0) + FX(1, 0) * FY(3, 0) + 2.0 * FX(2, 0) * FY(2, 0);
    R[1] = FX(3, 2) * FY(1, 0) + FX(1, 2) * FY(3, 0) + 2.0 * FX(2, 2) * FY(2, 0);
    R[2] = FX(3, 1) * FY(1, 1) + FX(1, 1) * FY(3, 1) + 2.0 * FX(2, 1) * FY(2, 1);
    R[3] = FX(3, 1) * FY(1, 0) + FX(1, 1) * FY(3, 0) + 2.0 * FX(2, 1) * FY(2, 0);
    R[4] = FX(3, 0) * FY(1, 2) + FX(1, 0) * FY(3, 2) + 2.0 * FX(2, 0) * FY(2, 2);
    R[5] = FX(3, 0) * FY(1, 1) + FX(1, 0) * FY(3, 1) + 2.0 * FX(2, 0) * FY(2, 1);
#undef FX
#undef FY
    R[0] = R[0] / ex1;
    R[1] = R[1] * ex1;
    R[2] = R[2] * ex1;
    R[4] = R[4] * ex1;
}

// W layout: [6][npts][NLAM], RC_* order, scaled by lambda and masked (calc_rc_tensor_module.F90:182-222)
__global__ void __launch_bounds__(256, 2) k_rc_weights(const VbtTab *__restrict__ T, int Nx, int Ny, double dx, double dy,
                                                    double xs, double ys, double *W)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *g = reinterpret_cast<double2 *>(smem_raw);  // [VN][6]
    // [NLAM][6] weights at the top of g: the normalisation reads only g[NFIRST*6 .. (NLAST+1)*6), below it
    static_assert((NLAST + 1) * 6 * sizeof(double2) <= VN * 6 * sizeof(double2) - NLAM * 6 * sizeof(double),
                  "weights would overlap the samples still being read");
    double *wt = reinterpret_cast<double *>(smem_raw + VN * 6 * sizeof(double2) - NLAM * 6 * sizeof(double));
    __shared__ double red[8], w0;
    const int Nx2 = 2 * Nx, Ny2 = 2 * Ny;
    const int pt = blockIdx.x, iy = pt / Nx2, ix = pt - iy * Nx2;
    const size_t npts = (size_t)Nx2 * Ny2;
    if (ix == Nx || iy == Ny) {  // lags Nx and Ny are zero (calc_rc_tensor_module.F90:84-92, :120-123)
        for (int k = threadIdx.x; k < NLAM; k += blockDim.x)
            for (int c = 0; c < 6; c++) W[((size_t)c * npts + pt) * NLAM + k] = 0.0;
        return;
    }
    const int lx = ix < Nx ? ix : ix - Nx2, ly = iy < Ny ? iy : iy - Ny2;
    // :190-193 and VBTransformWeightsAllSingleInt (VolumeBesselTransforms.F90:198-229)
    const double x = lx * dx - dx / 2.0 + xs, y = ly * dy - dy / 2.0 + ys;
    const double rho = sqrt(x * x + y * y);
    const double alpha = dx / rho, beta = dy / rho, phi = atan2(y, x);
    const double cphi = cos(phi), sphi = sin(phi), s_arg = log(rho) - T->lambda_shift;
    for (int i = threadIdx.x; i < VN; i += blockDim.x) {
        double R[6];
        outfunc2(i, s_arg, cphi, sphi, alpha, beta, R);
        const double sg = (i & 1) ? -1.0 : 1.0;
        const int p = T->inds[i];
        for (int c = 0; c < 6; c++) g[p * 6 + c] = make_double2(sg * R[c], 0.0);
    }
    __syncthreads();
    vbt_weights22(g, T);
    // normalisation (:282-285), real part for k in [NFIRST, NLAST], the rho factors of the single
    // integral (:224-228), and the column order of :194-199
    const int colmap[6] = {RC_D0, RC_DXX, RC_DXY, RC_DX, RC_DYY, RC_DY};
    double mx = 0.0;
    for (int k = threadIdx.x; k < NLAM; k += blockDim.x) {
        const int idx = k + NFIRST;
        const double sg = (idx & 1) ? -1.0 : 1.0;
        for (int c = 0; c < 6; c++) {
            double v = sg * g[idx * 6 + c].x / (double)VN;
            v = (c == 0) ? v * rho : ((c == 3 || c == 5) ? v : v / rho);
            wt[k * 6 + colmap[c]] = v;
            mx = fmax(mx, fabs(v));
        }
    }
    // W0 = MAXVAL(ABS(WT)) over all lambdas and columns (:200)
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
        w0 = m;
    }
    __syncthreads();
    // threshold (:207-209) and lambda scalings (:210-216)
    for (int k = threadIdx.x; k < NLAM; k += blockDim.x) {
        double mxr = 0.0;
        for (int c = 0; c < 6; c++) mxr = fmax(mxr, fabs(wt[k * 6 + c] / w0));
        const bool keep = mxr > WT_THRESHOLD;
        const double lm = T->lms[k];
        double v[6];
        v[RC_DXX] = wt[k * 6 + RC_DXX] / lm;
        v[RC_DYY] = wt[k * 6 + RC_DYY] / lm;
        v[RC_DXY] = wt[k * 6 + RC_DXY] / lm;
        v[RC_DX] = wt[k * 6 + RC_DX] * lm;
        v[RC_DY] = wt[k * 6 + RC_DY] * lm;
        v[RC_D0] = wt[k * 6 + RC_D0] * lm;
        for (int c = 0; c < 6; c++) W[((size_t)c * npts + pt) * NLAM + k] = keep ? v[c] : 0.0;
    }
}

// ---- 2-D FFT passes over [rows][Nx2][E] point-major buffers -----------------------------------------
enum { PASS_GENERIC = 0, PASS_CURRENTS = 1, PASS_FIELDS = 2 };

struct PassArgs {
    const double2 *in;   // GENERIC / FIELDS: [pts][E]; CURRENTS: the field E [3][Nz][Ny][Nx]
    double2 *out;        // GENERIC / CURRENTS: [pts][E]; FIELDS: Ea
    double2 *out2;       // FIELDS: Ha
    const double2 *dsig; // CURRENTS: csiga - csigb, [Nz][Ny][Nx]
    const double2 *tw;   // exp(-2 pi i j / L), j < L/2
    int L, lg;           // line length (power of two) and log2
    int E;               // elements per point
    int TE;              // elements per CTA tile
    int line_stride, elem_stride;  // point index = line * line_stride + i * elem_stride
    int nload, nstore;   // positions loaded (rest zero) and stored
    int Nx, Ny, Nz, Nr;
    int inverse;
    double scale;        // FIELDS: 1 / (4 Nx Ny) as a divisor
};

template <int MODE>
__global__ void __launch_bounds__(256) k_rc_pass(PassArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *s = reinterpret_cast<double2 *>(smem_raw);  // [L][TE]
    const int TE = a.TE, line = blockIdx.x, e0 = blockIdx.y * TE;
    const int ne = min(TE, a.E - e0);
    for (int i = threadIdx.x; i < a.L * TE; i += blockDim.x) s[i] = make_double2(0.0, 0.0);
    __syncthreads();
    if (MODE == PASS_CURRENTS) {
        // LoadEint (Continuation_Function_Module.F90:240-263): j = (csiga - csigb) E, row y = line, x fastest
        const size_t cells = (size_t)a.Nx * a.Ny * a.Nz;
        for (int i = threadIdx.x; i < a.nload * TE; i += blockDim.x) {
            const int t = i / a.nload, x = i - t * a.nload;
            if (t >= ne) continue;
            const int e = e0 + t, c = e / a.Nz, z = e - c * a.Nz;
            const size_t cell = ((size_t)z * a.Ny + line) * a.Nx + x;
            s[bitrev(x, a.lg) * TE + t] = cmul(a.dsig[cell], a.in[(size_t)c * cells + cell]);
        }
    } else {
        for (int i = threadIdx.x; i < a.nload * TE; i += blockDim.x) {
            const int x = i / TE, t = i - x * TE;
            if (t >= ne) continue;
            const size_t pt = (size_t)line * a.line_stride + (size_t)x * a.elem_stride;
            s[bitrev(x, a.lg) * TE + t] = a.in[pt * a.E + e0 + t];
        }
    }
    __syncthreads();
    smem_fft<double2, true>(s, a.lg, TE, 1, TE, a.tw, a.inverse != 0);
    if (MODE == PASS_FIELDS) {
        // x < Nx of row y = line, divided by 4 Nx Ny; element e = (f * 3 + c) * Nr + r
        const int half = 3 * a.Nr;
        for (int i = threadIdx.x; i < a.nstore * TE; i += blockDim.x) {
            const int x = i / TE, t = i - x * TE;
            if (t >= ne) continue;
            const int e = e0 + t, f = e / half, cr = e - f * half;
            const double2 v = s[x * TE + t];
            double2 *dst = f ? a.out2 : a.out;
            dst[((size_t)line * a.Nx + x) * half + cr] = make_double2(v.x / a.scale, v.y / a.scale);
        }
    } else {
        for (int i = threadIdx.x; i < a.nstore * TE; i += blockDim.x) {
            const int x = i / TE, t = i - x * TE;
            if (t >= ne) continue;
            const size_t pt = (size_t)line * a.line_stride + (size_t)x * a.elem_stride;
            a.out[pt * a.E + e0 + t] = s[x * TE + t];
        }
    }
}

// ---- contraction at every spectral point -------------------------------------------------------------
// APPLY_RC_E_OP / APPLY_RC_H_OP (Continuation_Function_Module.F90:382-481): per point and receiver
//   Ex = XX jx + XY jy + XZ jz    Ey = XY jx + YY jy + YZ jz    Ez = ZX jx + ZY jy + ZZ jz
//   Hx = HXX jx + HXY jy + HXZ jz Hy = HYX jx - HXX jy + HYZ jz Hz = HZX jx + HZY jy
// each term a sum over z (ZGEMV('T')).  One warp per point, lanes over z (Nz <= 64).
__global__ void __launch_bounds__(256) k_rc_contract(const double2 *__restrict__ G, const double2 *__restrict__ U,
                                                     double2 *__restrict__ O, long long npts, int Nr, int Nz)
{
    const int lane = threadIdx.x & 31;
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const size_t E = (size_t)RC_NCOMP * Nr * Nz;
    for (long long p = warp; p < npts; p += nwarps) {
        const double2 *u = U + (size_t)p * 3 * Nz;
        double2 ux[2], uy[2], uz[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int z = lane + 32 * k;
            const bool ok = z < Nz;
            ux[k] = ok ? u[z] : make_double2(0.0, 0.0);
            uy[k] = ok ? u[Nz + z] : make_double2(0.0, 0.0);
            uz[k] = ok ? u[2 * Nz + z] : make_double2(0.0, 0.0);
        }
        const double2 *g = G + (size_t)p * E;
        for (int r = 0; r < Nr; r++) {
            double2 acc[6];
#pragma unroll
            for (int o = 0; o < 6; o++) acc[o] = make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int z = lane + 32 * k;
                if (z >= Nz) continue;
                auto gc = [&](int c) { return g[((size_t)c * Nr + r) * Nz + z]; };
                cfma(acc[0], gc(REXX), ux[k]);
                cfma(acc[0], gc(REXY), uy[k]);
                cfma(acc[0], gc(REXZ), uz[k]);
                cfma(acc[1], gc(REXY), ux[k]);
                cfma(acc[1], gc(REYY), uy[k]);
                cfma(acc[1], gc(REYZ), uz[k]);
                cfma(acc[2], gc(REZX), ux[k]);
                cfma(acc[2], gc(REZY), uy[k]);
                cfma(acc[2], gc(REZZ), uz[k]);
                const double2 hxx = gc(RHXX);
                cfma(acc[3], hxx, ux[k]);
                cfma(acc[3], gc(RHXY), uy[k]);
                cfma(acc[3], gc(RHXZ), uz[k]);
                cfma(acc[4], gc(RHYX), ux[k]);
                cfma(acc[4], make_double2(-hxx.x, -hxx.y), uy[k]);
                cfma(acc[4], gc(RHYZ), uz[k]);
                cfma(acc[5], gc(RHZX), ux[k]);
                cfma(acc[5], gc(RHZY), uy[k]);
            }
#pragma unroll
            for (int o = 0; o < 6; o++)
                for (int sh = 16; sh > 0; sh >>= 1) {
                    acc[o].x += __shfl_xor_sync(0xffffffffu, acc[o].x, sh);
                    acc[o].y += __shfl_xor_sync(0xffffffffu, acc[o].y, sh);
                }
            if (lane < 6) {
                double2 v = acc[0];
#pragma unroll
                for (int o = 1; o < 6; o++)
                    if (lane == o) v = acc[o];
                O[((size_t)p * 6 + lane) * Nr + r] = v;
            }
        }
    }
}

void make_twiddles(std::vector<double2> &tw, int L)
{
    tw.resize(L / 2);
    const double pi = 3.14159265358979323846264338327950288;
    for (int j = 0; j < L / 2; j++) {
        const double th = -2.0 * pi * j / L;
        tw[j] = make_double2(std::cos(th), std::sin(th));
    }
}

int pass_tile(int L)
{
    int te = 16;
    while (te > 1 && (size_t)L * te * sizeof(double2) > 131072) te /= 2;
    return te;
}

}  // namespace

struct RcOp {
    int Nx = 0, Ny = 0, Nz = 0, Nr = 0;
    double dx = 0, dy = 0;
    std::vector<double> z;
    std::vector<RcReceiver> recv;
    bool have_tensor = false, have_spectral = false, have_sigma = false, have_background = false;
    double2 *d_G = nullptr;     // [2Ny][2Nx][15][Nr][Nz]
    double2 *d_U = nullptr;     // [2Ny][2Nx][3Nz]
    double2 *d_O = nullptr;     // [2Ny][2Nx][6Nr]
    double2 *d_csiga = nullptr; // [Nz][Ny][Nx]
    double2 *d_dsig = nullptr;  // csiga - csigb
    double2 *d_twx = nullptr, *d_twy = nullptr;
    double2 *d_E = nullptr, *d_Ea = nullptr, *d_Ha = nullptr;  // staging of the host-buffer entry
    std::vector<double2> csigb;  // per cell
    cudaStream_t stream = nullptr;

    size_t npts() const { return (size_t)4 * Nx * Ny; }
    size_t E() const { return (size_t)RC_NCOMP * Nr * Nz; }
    size_t cells() const { return (size_t)Nx * Ny * Nz; }
};

#define RC_TRY(expr)                                                  \
    do {                                                              \
        cudaError_t e_ = (expr);                                      \
        if (e_ != cudaSuccess) {                                      \
            g2_set_error(__FILE__, __LINE__, cudaGetErrorString(e_)); \
            return G2_ERR_CUDA;                                       \
        }                                                             \
    } while (0)

RcOp *rc_create(int Nx, int Ny, int Nz, double dx, double dy, const double *z, int Nr, const RcReceiver *recv)
{
    RcOp *op = new RcOp();
    op->Nx = Nx;
    op->Ny = Ny;
    op->Nz = Nz;
    op->Nr = Nr;
    op->dx = dx;
    op->dy = dy;
    op->z.assign(z, z + Nz + 1);
    op->recv.assign(recv, recv + Nr);
    bool ok = cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&op->d_G, op->npts() * op->E() * sizeof(double2)) == cudaSuccess;
    ok = ok && cudaMalloc(&op->d_U, op->npts() * 3 * Nz * sizeof(double2)) == cudaSuccess;
    ok = ok && cudaMalloc(&op->d_O, op->npts() * 6 * Nr * sizeof(double2)) == cudaSuccess;
    ok = ok && cudaMalloc(&op->d_csiga, op->cells() * sizeof(double2)) == cudaSuccess;
    ok = ok && cudaMalloc(&op->d_dsig, op->cells() * sizeof(double2)) == cudaSuccess;
    std::vector<double2> tw;
    if (ok) {
        make_twiddles(tw, 2 * Nx);
        ok = cudaMalloc(&op->d_twx, tw.size() * sizeof(double2)) == cudaSuccess &&
             cudaMemcpyAsync(op->d_twx, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, op->stream) ==
                 cudaSuccess &&
             cudaStreamSynchronize(op->stream) == cudaSuccess;
    }
    if (ok) {
        make_twiddles(tw, 2 * Ny);
        ok = cudaMalloc(&op->d_twy, tw.size() * sizeof(double2)) == cudaSuccess &&
             cudaMemcpyAsync(op->d_twy, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, op->stream) ==
                 cudaSuccess &&
             cudaStreamSynchronize(op->stream) == cudaSuccess;
    }
    if (!ok) {
        g2_set_error_msg("rc_create: device allocation failed");
        rc_delete(op);
        return nullptr;
    }
    return op;
}

void rc_delete(RcOp *op)
{
    if (!op) return;
    if (op->stream) cudaStreamSynchronize(op->stream);
    void *ptrs[] = {op->d_G, op->d_U, op->d_O, op->d_csiga, op->d_dsig, op->d_twx, op->d_twy,
                    op->d_E, op->d_Ea, op->d_Ha};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (op->stream) cudaStreamDestroy(op->stream);
    delete op;
}

int rc_count(const RcOp *op) { return op->Nr; }
int rc_nz(const RcOp *op) { return op->Nz; }
const double *rc_borders(const RcOp *op) { return op->z.data(); }
cudaStream_t rc_stream(const RcOp *op) { return op->stream; }
int rc_receivers(const RcOp *op, RcReceiver *out)
{
    std::memcpy(out, op->recv.data(), sizeof(RcReceiver) * op->recv.size());
    return G2_OK;
}

static int rc_update_dsig(RcOp *op)
{
    if (!op->have_sigma || !op->have_background) return G2_OK;
    // dsig = csiga - csigb(z) (LoadEint :254), computed on the host once per conductivity / frequency
    std::vector<double2> h(op->cells());
    RC_TRY(cudaMemcpyAsync(h.data(), op->d_csiga, h.size() * sizeof(double2), cudaMemcpyDeviceToHost, op->stream));
    RC_TRY(cudaStreamSynchronize(op->stream));
    const size_t plane = (size_t)op->Nx * op->Ny;
    for (int iz = 0; iz < op->Nz; iz++)
        for (size_t k = 0; k < plane; k++) {
            double2 &v = h[iz * plane + k];
            v = make_double2(v.x - op->csigb[iz].x, v.y - op->csigb[iz].y);
        }
    RC_TRY(cudaMemcpyAsync(op->d_dsig, h.data(), h.size() * sizeof(double2), cudaMemcpyHostToDevice, op->stream));
    RC_TRY(cudaStreamSynchronize(op->stream));
    return G2_OK;
}

int rc_set_anomaly_conductivity(RcOp *op, const double2 *csiga_host)
{
    RC_TRY(cudaMemcpyAsync(op->d_csiga, csiga_host, op->cells() * sizeof(double2), cudaMemcpyHostToDevice, op->stream));
    RC_TRY(cudaStreamSynchronize(op->stream));
    op->have_sigma = true;
    return rc_update_dsig(op);
}

int rc_calc_kernel(RcOp *op, int Nl, const double2 *csigma, const double *thick, double omega, const int *Lnumber)
{
    const int Nx = op->Nx, Ny = op->Ny, Nz = op->Nz, Nr = op->Nr;
    if (Nl < 1 || Nl > MAXL || Nz > MAXZ) {
        g2_set_error_msg("receiver tensor on the GPU supports up to 16 layers and Nz <= 64");
        return G2_ERR_UNSUPPORTED;
    }
    cudaStream_t st = op->stream;
    Bkg h{};
    h.Nl = Nl;
    h.Nz = Nz;
    const double mu0 = 4.0 * PI_D * 1e-7;
    for (int i = 0; i <= Nl; i++) {
        h.csigma[i] = csigma[i];
        // SET_FREQ / CREATE_BACKGROUND: k2 = i csigma mu0 omega
        h.k2[i] = make_double2(-csigma[i].y * mu0 * omega, csigma[i].x * mu0 * omega);
    }
    for (int i = 1; i <= Nl - 1; i++) h.thick[i] = thick[i - 1];
    if (Nl > 1) {
        h.depth[1] = h.thick[1];
        for (int i = 2; i <= Nl - 1; i++) h.depth[i] = h.depth[i - 1] + h.thick[i];
    }
    h.iwm = make_double2(0.0, mu0 * omega);
    for (int i = 0; i <= Nz; i++) {
        h.L[i] = Lnumber[i];
        h.z[i] = op->z[i];
    }
    for (int i = 1; i <= Nz; i++) h.dz[i] = op->z[i] - op->z[i - 1];
    op->csigb.resize(Nz);
    for (int iz = 1; iz <= Nz; iz++) op->csigb[iz - 1] = csigma[Lnumber[iz]];  // FinalizeRCOperator :178-181
    std::vector<RcRecvDev> rv(Nr);
    for (int r = 0; r < Nr; r++) rv[r] = RcRecvDev{op->recv[r].zrecv, op->recv[r].recv_layer, op->recv[r].anom_cell};
    VbtTab *tab = new VbtTab();
    // VBTransformInit(rmin) with rmin = sqrt(dx^2 + dy^2) / 2 (calc_rc_tensor_module.F90:79-80)
    make_vbt(std::sqrt(op->dx * op->dx + op->dy * op->dy) / 2.0, *tab);

    Bkg *d_bkg = nullptr;
    VbtTab *d_tab = nullptr;
    RcRecvDev *d_rv = nullptr;
    double2 *d_B = nullptr;
    double *d_W = nullptr;
    const size_t npts = op->npts();
    int rc = G2_OK;
    auto cleanup = [&]() {
        cudaFree(d_bkg);
        cudaFree(d_tab);
        cudaFree(d_rv);
        cudaFree(d_B);
        cudaFree(d_W);
        delete tab;
    };
#define RC_TRY2(expr)                                                     \
    do {                                                                  \
        cudaError_t e_ = (expr);                                          \
        if (e_ != cudaSuccess) {                                          \
            g2_set_error(__FILE__, __LINE__, cudaGetErrorString(e_));     \
            cleanup();                                                    \
            return G2_ERR_CUDA;                                           \
        }                                                                 \
    } while (0)
    RC_TRY2(cudaMalloc(&d_bkg, sizeof(Bkg)));
    RC_TRY2(cudaMalloc(&d_tab, sizeof(VbtTab)));
    RC_TRY2(cudaMalloc(&d_rv, sizeof(RcRecvDev) * Nr));
    RC_TRY2(cudaMemcpyAsync(d_bkg, &h, sizeof(Bkg), cudaMemcpyHostToDevice, st));
    RC_TRY2(cudaMemcpyAsync(d_tab, tab, sizeof(VbtTab), cudaMemcpyHostToDevice, st));
    RC_TRY2(cudaMemcpyAsync(d_rv, rv.data(), sizeof(RcRecvDev) * Nr, cudaMemcpyHostToDevice, st));
    RC_TRY2(cudaMalloc(&d_B, sizeof(double2) * (size_t)Nr * RC_NBASIS * NLAM * Nz));
    RC_TRY2(cudaMalloc(&d_W, sizeof(double) * 6 * npts * NLAM));
    double *d_lms = reinterpret_cast<double *>(reinterpret_cast<char *>(d_tab) + offsetof(VbtTab, lms));
    k_rc_basis<<<dim3(NLAM, Nr), 64, 0, st>>>(d_bkg, d_rv, d_lms, d_B);
    RC_TRY2(cudaGetLastError());
    const size_t smw = sizeof(double2) * VN * 6;  // two blocks per SM
    RC_TRY2(cudaFuncSetAttribute(k_rc_weights, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw));
    const double sc = 1.0 / 4.0 / PI_D;  // s = 1/4/PI (calc_rc_tensor_module.F90:184), G * s (:225-226)
    const int E = (int)op->E();
    const int gm = (int)((npts + GM - 1) / GM);
    int launches = 1;
    for (int r = 0; r < Nr; r++) {
        k_rc_weights<<<(unsigned)npts, 256, smw, st>>>(d_tab, Nx, Ny, op->dx, op->dy, op->recv[r].x_shift,
                                                        op->recv[r].y_shift, d_W);
        RC_TRY2(cudaGetLastError());
        auto Wt = [&](int c) { return d_W + (size_t)c * npts * NLAM; };
        auto Bs = [&](int bsel) { return d_B + ((size_t)r * RC_NBASIS + bsel) * NLAM * Nz; };
        auto gemm = [&](int comp, int w1, int b1, int w2, int b2) {
            dim3 grid(gm, (Nz + GN - 1) / GN);
            k_gemm<<<grid, 256, 0, st>>>(Wt(w1), Bs(b1), w2 >= 0 ? Wt(w2) : nullptr, w2 >= 0 ? Bs(b2) : nullptr,
                                         (int)npts, Nz, op->d_G, E, (comp * Nr + r) * Nz, sc);
        };
        // rc_kernel_hankel_module.F90:118-143
        gemm(REXX, RC_D0, B_G11, RC_DXX, B_G3DZ_G11);
        gemm(REXY, RC_DXY, B_G3DZ_G11, -1, 0);
        gemm(REXZ, RC_DX, B_G2DZ, -1, 0);
        gemm(REYY, RC_D0, B_G11, RC_DYY, B_G3DZ_G11);
        gemm(REYZ, RC_DY, B_G2DZ, -1, 0);
        gemm(REZX, RC_DX, B_G2DZ0, -1, 0);
        gemm(REZY, RC_DY, B_G2DZ0, -1, 0);
        gemm(REZZ, RC_D0, B_G2G2DZZ, -1, 0);
        gemm(RHXX, RC_DXY, B_G3, -1, 0);
        gemm(RHXY, RC_DYY, B_G3, RC_D0, B_MG1DZ);
        gemm(RHXZ, RC_DY, B_G2, -1, 0);
        gemm(RHYX, RC_D0, B_G1DZ, RC_DXX, B_MG3);
        gemm(RHYZ, RC_DX, B_MG2, -1, 0);
        gemm(RHZX, RC_DY, B_MG1, -1, 0);
        gemm(RHZY, RC_DX, B_G1, -1, 0);
        RC_TRY2(cudaGetLastError());
        launches += 1 + RC_NCOMP;
    }
    RC_TRY2(cudaStreamSynchronize(st));
    g2_count_launches(launches);
    cleanup();
#undef RC_TRY2
    op->have_tensor = true;
    op->have_spectral = false;
    op->have_background = true;
    rc = rc_update_dsig(op);
    return rc;
}

static int launch_pass(int mode, const PassArgs &a, int nlines, cudaStream_t st)
{
    const size_t sm = (size_t)a.L * a.TE * sizeof(double2);
    dim3 grid(nlines, (a.E + a.TE - 1) / a.TE);
    switch (mode) {
    case PASS_GENERIC:
        RC_TRY(cudaFuncSetAttribute(k_rc_pass<PASS_GENERIC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_rc_pass<PASS_GENERIC><<<grid, 256, sm, st>>>(a);
        break;
    case PASS_CURRENTS:
        RC_TRY(cudaFuncSetAttribute(k_rc_pass<PASS_CURRENTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_rc_pass<PASS_CURRENTS><<<grid, 256, sm, st>>>(a);
        break;
    default:
        RC_TRY(cudaFuncSetAttribute(k_rc_pass<PASS_FIELDS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_rc_pass<PASS_FIELDS><<<grid, 256, sm, st>>>(a);
        break;
    }
    RC_TRY(cudaGetLastError());
    return G2_OK;
}

static PassArgs base_args(const RcOp *op, bool along_x, int E)
{
    PassArgs a{};
    a.L = along_x ? 2 * op->Nx : 2 * op->Ny;
    a.lg = ilog2(a.L);
    a.tw = along_x ? op->d_twx : op->d_twy;
    a.E = E;
    a.TE = pass_tile(a.L);
    // rows: point = line * 2Nx + i; columns: point = i * 2Nx + line
    a.line_stride = along_x ? 2 * op->Nx : 1;
    a.elem_stride = along_x ? 1 : 2 * op->Nx;
    a.nload = a.nstore = a.L;
    a.Nx = op->Nx;
    a.Ny = op->Ny;
    a.Nz = op->Nz;
    a.Nr = op->Nr;
    a.scale = 1.0;
    return a;
}

int rc_fft_kernel(RcOp *op)
{
    if (!op->have_tensor) {
        g2_set_error_msg("rc_fft_kernel: no receiver tensor (compute it first)");
        return G2_ERR_STATE;
    }
    if (op->have_spectral) return G2_OK;
    const int E = (int)op->E();
    PassArgs a = base_args(op, true, E);  // CalcFFTofRCTensor (:330-366): forward 2-D FFT, in place
    a.in = a.out = op->d_G;
    int rc = launch_pass(PASS_GENERIC, a, 2 * op->Ny, op->stream);
    if (rc) return rc;
    PassArgs b = base_args(op, false, E);
    b.in = b.out = op->d_G;
    rc = launch_pass(PASS_GENERIC, b, 2 * op->Nx, op->stream);
    if (rc) return rc;
    RC_TRY(cudaStreamSynchronize(op->stream));
    g2_count_launches(2);
    op->have_spectral = true;
    return G2_OK;
}

int rc_recalculate_device(RcOp *op, const double2 *dE, double2 *dEa, double2 *dHa)
{
    if (!op->have_spectral || !op->have_sigma) {
        g2_set_error_msg("rc_recalculate: needs the transformed receiver tensor and the anomaly conductivity");
        return G2_ERR_STATE;
    }
    const int Nx = op->Nx, Ny = op->Ny, Nz = op->Nz, Nr = op->Nr;
    cudaStream_t st = op->stream;
    // forward: currents along x (rows y < Ny), then y (rows >= Ny are zero)
    PassArgs a = base_args(op, true, 3 * Nz);
    a.in = dE;
    a.dsig = op->d_dsig;
    a.out = op->d_U;
    a.nload = Nx;
    int rc = launch_pass(PASS_CURRENTS, a, Ny, st);
    if (rc) return rc;
    PassArgs b = base_args(op, false, 3 * Nz);
    b.in = b.out = op->d_U;
    b.nload = Ny;
    rc = launch_pass(PASS_GENERIC, b, 2 * Nx, st);
    if (rc) return rc;
    const long long npts = (long long)op->npts();
    int nsm = 148;
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    const long long blocks = std::min<long long>((npts + 7) / 8, (long long)nsm * 8);
    k_rc_contract<<<(unsigned)blocks, 256, 0, st>>>(op->d_G, op->d_U, op->d_O, npts, Nr, Nz);
    RC_TRY(cudaGetLastError());
    // inverse: y (keep rows < Ny), then x (keep x < Nx) into Ea / Ha
    PassArgs c = base_args(op, false, 6 * Nr);
    c.in = c.out = op->d_O;
    c.inverse = 1;
    c.nstore = Ny;
    rc = launch_pass(PASS_GENERIC, c, 2 * Nx, st);
    if (rc) return rc;
    PassArgs d = base_args(op, true, 6 * Nr);
    d.in = op->d_O;
    d.out = dEa;
    d.out2 = dHa;
    d.inverse = 1;
    d.nstore = Nx;
    d.scale = (double)(4 * (long long)Nx * Ny);
    rc = launch_pass(PASS_FIELDS, d, Ny, st);
    if (rc) return rc;
    g2_count_launches(5);
    return G2_OK;
}

int rc_recalculate_host(RcOp *op, const double2 *E, double2 *Ea, double2 *Ha)
{
    const size_t nE = 3 * op->cells(), nF = (size_t)op->Nx * op->Ny * 3 * op->Nr;
    if (!op->d_E) {
        RC_TRY(cudaMalloc(&op->d_E, nE * sizeof(double2)));
        RC_TRY(cudaMalloc(&op->d_Ea, nF * sizeof(double2)));
        RC_TRY(cudaMalloc(&op->d_Ha, nF * sizeof(double2)));
    }
    RC_TRY(cudaMemcpyAsync(op->d_E, E, nE * sizeof(double2), cudaMemcpyHostToDevice, op->stream));
    int rc = rc_recalculate_device(op, op->d_E, op->d_Ea, op->d_Ha);
    if (rc) return rc;
    RC_TRY(cudaMemcpyAsync(Ea, op->d_Ea, nF * sizeof(double2), cudaMemcpyDeviceToHost, op->stream));
    RC_TRY(cudaMemcpyAsync(Ha, op->d_Ha, nF * sizeof(double2), cudaMemcpyDeviceToHost, op->stream));
    RC_TRY(cudaStreamSynchronize(op->stream));
    return G2_OK;
}

int rc_copy_kernel(RcOp *op, double2 *host)
{
    if (!op->have_tensor) {
        g2_set_error_msg("rc_copy_kernel: no receiver tensor");
        return G2_ERR_STATE;
    }
    RC_TRY(cudaMemcpyAsync(host, op->d_G, op->npts() * op->E() * sizeof(double2), cudaMemcpyDeviceToHost, op->stream));
    RC_TRY(cudaStreamSynchronize(op->stream));
    return G2_OK;
}
