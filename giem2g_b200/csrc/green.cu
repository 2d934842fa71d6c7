// Spatial Green's tensor of the contracting IE on the GPU, FP64.
//
// Restates CalcIntegralGreenTensor (calc_ie_tensor_module.F90:54-293) with its helpers
// ie_kernel_hankel_module.F90 (Calc_Double_Integral_U, GoByShellsU/L), apq_module.F90 (Calc_APQ,
// frames, Calc_FtFb) and VolumeBesselTransforms.F90 (VBTransformInit, weights by FFT deconvolution).
//
// The reference loops over lags (lx,ly), builds the lag's Hankel weights WT(lambda, 6) and then, for
// every lambda whose weights pass the 1e-12 threshold, runs the layered-medium recursion and the shell
// sweeps.  Everything in that inner part except the six weights is independent of the lag, and the
// accumulation is linear in the weights.  So the GPU computes
//   (1) k_basis:   per lambda, four Nz x Nz basis matrices M1..M4 (the shell products of GoByShellsU/L
//                  and the diagonal terms), once for all lags;
//   (2) k_weights: per lag, the 501 x 6 weights (1024-point FFT deconvolution in shared memory), the
//                  COMPUTE_WEIGHTS zeroing, the threshold mask and the lambda scalings;
//   (3) k_gemm:    G_c(lag) = sum_lambda sum_w W_w(lag, lambda) M_{c,w}(lambda):
//                    xx = D0*M1 + DXX*M2, yy = D0*M1 + DYY*M2, xy = DXY*M2, xz = DX*M3, yz = DY*M3,
//                    zz = D0*M4, all divided by 4 pi.
// A lambda that the reference skips for a lag has all six weights zero here, so the sums hold the
// same terms; only the order of the floating-point additions differs.
#include <cmath>
#include <vector>
#include <cuda/std/complex>
#include "common.cuh"
#include "ie_internal.h"
#include "hankel.cuh"

namespace {

enum { IE_DXX = 0, IE_DXY = 1, IE_DYY = 2, IE_DX = 3, IE_DY = 4, IE_D0 = 5 };

// ---- (1) lambda basis ---------------------------------------------------------------------------
// Bas layout: M1,M2,M4 packed upper [NLAM][P]; M3 full column-major [NLAM][Nz*Nz].
__global__ void k_basis(const Bkg *__restrict__ bk, const double *__restrict__ lms_all, double2 *M1, double2 *M2,
                        double2 *M3, double2 *M4)
{
    const int li = blockIdx.x;
    const double lms = lms_all[li];
    const Bkg &b = *bk;
    const int Nz = b.Nz, P = Nz * (Nz + 1) / 2;
    __shared__ cplx fc1[MAXZ + 1], fc2[MAXZ + 1], tf1[MAXZ + 1], tf2[MAXZ + 1], tf3[MAXZ + 1];
    __shared__ cplx fcb[MAXZ + 1], bfr[MAXZ + 1], Ft1[MAXZ + 1], Ft2[MAXZ + 1], Ft3[MAXZ + 1], Fb[MAXZ + 1];
    __shared__ cplx G1[MAXZ + 1], G2_[MAXZ + 1], G3[MAXZ + 1], G4[MAXZ + 1];
    if (threadIdx.x == 0) {
        // Calc_Apq (apq_module.F90:230-266)
        cplx eta[MAXL + 1], el[MAXL + 1], p[MAXL + 1][2], q[MAXL + 1][2], Arr[MAXL + 1][2];
        dev_apq(b, lms, eta, el, p, q, Arr);
        // expz (ie_kernel_hankel_module.F90:69-72), pexpz (apq_module.F90:112-137), qexpz (:155-177)
        cplx expz[MAXZ + 1], pez[MAXZ + 1][2], qez[MAXZ + 1][2];
        for (int iz = 1; iz <= Nz; iz++) expz[iz] = cuda::std::exp(-eta[b.L[iz]] * b.dz[iz]);
        dev_pexpz(b, eta, p, expz, pez);
        dev_qexpz(b, eta, q, expz, qez);
        // Calc_tframe_p (apq_module.F90:83-110)
        for (int i = 1; i <= Nz - 1; i++) {
            const int l = b.L[i];
            cplx a[2], bb[2], c[2];
            for (int k = 0; k < 2; k++) {
                a[k] = pez[i][k];
                bb[k] = a[k] * expz[i];
                c[k] = bb[k] * expz[i];
                a[k] = 1.0 + a[k];
                bb[k] = 1.0 + bb[k];
                c[k] = 1.0 + c[k];
            }
            const cplx w = (1.0 - expz[i]) / eta[l];
            fc1[i] = expz[i] * a[0] / c[0];
            fc2[i] = expz[i] * a[1] / c[1];
            tf1[i] = w * bb[0] / c[0];
            tf2[i] = (1.0 - fc2[i]) / C(b.csigma[l]);
            tf3[i] = (w * bb[1] / c[1]) / C(b.csigma[l]);
        }
        // Calc_bframe_q (apq_module.F90:138-153)
        for (int i = Nz; i >= 2; i--) {
            const int l = b.L[i];
            cplx a = qez[i][1];
            const cplx d = 1.0 + a * expz[i] * expz[i];
            a = 1.0 + a;
            fcb[i] = expz[i] * a / d;
            bfr[i] = (fcb[i] - 1.0) / C(b.csigma[l]);
        }
        // Calc_FtFb (apq_module.F90:31-79)
        for (int i = 1; i <= Nz; i++) {
            const int l = b.L[i];
            cplx a[2], a1[2], a2[2], p1[2], p2[2], pe1[2], pe2[2], q1[2], q2[2], qe1[2], qe2[2], w[2], Fb3[3];
            for (int k = 0; k < 2; k++) {
                a[k] = (1.0 - expz[i]) * Arr[l][k];
                a1[k] = a[k] / eta[l];
                a2[k] = a1[k] / eta[l];
                p1[k] = 1.0 + pez[i][k];
                p2[k] = 1.0 - pez[i][k];
                pe1[k] = 1.0 + pez[i][k] * expz[i];
                pe2[k] = -1.0 + pez[i][k] * expz[i];
                q1[k] = 1.0 + qez[i][k];
                q2[k] = 1.0 - qez[i][k];
                qe1[k] = 1.0 + qez[i][k] * expz[i];
                qe2[k] = 1.0 - qez[i][k] * expz[i];
            }
            const cplx eta2 = eta[l] * eta[l];
            const cplx ft1 = a1[0] * p1[0] * qe1[0], ft2 = a1[1] * p1[1] * qe1[1], ft3 = a[1] * p1[1] * qe2[1];
            Fb3[0] = a1[0] * pe1[0] * q1[0];
            Fb3[1] = a1[1] * pe1[1] * q1[1];
            Fb3[2] = a[1] * pe2[1] * q1[1];
            for (int k = 0; k < 2; k++) w[k] = -a2[k] * (p2[k] * qe1[k] + pe1[k] * q2[k]);
            const double dzi = b.dz[i];
            G1[i] = w[0] + 2.0 / eta2 * dzi;
            G2_[i] = Fb3[1] - ft2;
            G3[i] = (w[1] + 2.0 / eta2 * dzi) * C(b.iwm) + eta2 / C(b.csigma[l]) * w[1];
            G4[i] = Fb3[2] - ft3 - eta2 * w[0];
            Ft1[i] = ft1;
            Ft2[i] = ft2;
            Ft3[i] = ft3;
            Fb[i] = Fb3[1];
        }
    }
    __syncthreads();
    // columns s (1-based source cell); shell products of GoByShellsU / GoByShellsL
    const double lm2 = lms * lms;
    const cplx iwm = C(b.iwm);
    for (int s = threadIdx.x + 1; s <= Nz; s += blockDim.x) {
        const int l = b.L[s];
        const cplx cs = C(b.csigma[l]);
        const size_t o1 = (size_t)li * P, o3 = (size_t)li * Nz * Nz;
        const int d = (s - 1) + (s - 1) * s / 2;  // packed (s-1, s-1)
        M1[o1 + d] = D2(G1[s] * iwm);
        M2[o1 + d] = D2((G1[s] * lm2 + G4[s]) / cs);
        M3[o3 + (s - 1) + (size_t)(s - 1) * Nz] = D2(G2_[s] / cs);
        M4[o1 + d] = D2(G3[s]);
        cplx t1 = Ft1[s] * iwm, t2 = Ft3[s], t3 = Ft2[s], t4 = Ft2[s] * lm2;
        for (int r = s - 1; r >= 1; r--) {
            const int pk = (r - 1) + (s - 1) * s / 2;  // packed (r-1, s-1), r < s
            const cplx a = t1 * tf1[r];
            M1[o1 + pk] = D2(a);
            M2[o1 + pk] = D2(a + t2 * tf2[r]);
            M3[o3 + (r - 1) + (size_t)(s - 1) * Nz] = D2(t3 * tf2[r]);
            M4[o1 + pk] = D2(t4 * tf3[r]);
            t1 = t1 * fc1[r];
            t2 = t2 * fc2[r];
            t3 = t3 * fc2[r];
            t4 = t4 * fc2[r];
        }
        cplx t5 = Fb[s];
        for (int r = s + 1; r <= Nz; r++) {
            M3[o3 + (r - 1) + (size_t)(s - 1) * Nz] = D2(t5 * bfr[r]);
            t5 = t5 * fcb[r];
        }
    }
}

// ---- (2) weights per lag -----------------------------------------------------------------------

G2_D void int2d(const double *x, const double *x2, const double *ex, const double *er, double R[3])
{
    double f[3];
    for (int k = 0; k < 3; k++) f[k] = x[k] * er[k];
    R[0] = (f[1] + f[2] - 2.0 * f[0]) * SPI * 0.25;
    for (int k = 0; k < 3; k++) f[k] = ex[k];
    R[1] = f[1] + f[2] - 2.0 * f[0];
    for (int k = 0; k < 3; k++) f[k] = ex[k] * x2[k] / 4.0;
    R[2] = f[1] + f[2] - 2.0 * f[0];
}
G2_D void dint_d0(const double *x, const double *x2, const double *ex, const double *er, double R[3])
{
    double f[3];
    int2d(x, x2, ex, er, f);
    R[0] = 32.0 * (1.5 * f[0] + f[1] + f[2]);
    R[1] = 8.0 * f[0] + 4.0 * f[1];
    R[2] = 4.0 * f[0] + f[1];
}
G2_D void dint_d1(const double *x, const double *x2, const double *ex, const double *er, double R[3])
{
    double f[3], g[3];
    for (int k = 0; k < 3; k++) g[k] = er[k];
    f[0] = (g[1] + g[2] - 2.0 * g[0]) * SPI * 0.5;
    for (int k = 0; k < 3; k++) g[k] = ex[k] * x[k];
    f[1] = g[1] + g[2] - 2.0 * g[0];
    for (int k = 0; k < 3; k++) g[k] = g[k] * x2[k];
    f[2] = g[1] + g[2] - 2.0 * g[0];
    R[0] = -8.0 * f[2] - 12.0 * f[1] + 12.0 * f[0];
    R[1] = -2.0 * f[1] + 2.0 * f[0];
    R[2] = f[0];
}
G2_D void dint_d2(const double *x2, const double *exv, double R[3])
{
    double ex[3], f[3];
    for (int k = 0; k < 3; k++) ex[k] = exv[k] / 2.0;
    for (int k = 0; k < 3; k++) f[k] = x2[k] * ex[k] * 4.0;
    R[1] = f[1] + f[2] - 2.0 * f[0];
    for (int k = 0; k < 3; k++) f[k] = x2[k] * f[k] * 4.0;
    R[0] = f[1] + f[2] - 2.0 * f[0];
    for (int k = 0; k < 3; k++) f[k] = ex[k];
    R[2] = f[1] + f[2] - 2.0 * f[0];
}

// VolumeBesselTransforms.F90:142-157, 304-340, 377-403 for sample i
G2_D void outfunc(int i, double s_arg, double cphi, double sphi, double alpha, double beta, double R[6])
{
    const int i0 = i & ~1;
    double y2 = (i0 + VN2) * Y_STEP + VP + s_arg;
    if (i & 1) y2 = y2 + Y_STEP;
    const double ex1 = exp(y2), ex2 = ex1 * ex1, ex3 = ex2 * ex1;
    double xv[3], yv[3], x2[3], yy2[3], xe[3], ye[3], xr[3], yr[3];
    {
        double x1 = ex1 * cphi, y1 = ex1 * sphi;
        const double dxv = alpha * ex1, dyv = beta * ex1;
        x1 = x1 - dxv * 0.5;
        y1 = y1 - dyv * 0.5;
        xv[0] = x1; xv[1] = x1 + dxv; xv[2] = x1 - dxv;
        yv[0] = y1; yv[1] = y1 + dyv; yv[2] = y1 - dyv;
        for (int k = 0; k < 3; k++) {
            xv[k] = xv[k] * 0.5;
            x2[k] = xv[k] * xv[k];
            xe[k] = exp(-x2[k]);
            xr[k] = erf(xv[k]);
            yv[k] = yv[k] * 0.5;
            yy2[k] = yv[k] * yv[k];
            ye[k] = exp(-yy2[k]);
            yr[k] = erf(yv[k]);
        }
    }
    double fx[3][3], fy[3][3];
    dint_d0(xv, x2, xe, xr, fx[0]);
    dint_d1(xv, x2, xe, xr, fx[1]);
    dint_d2(x2, xe, fx[2]);
    dint_d0(yv, yy2, ye, yr, fy[0]);
    dint_d1(yv, yy2, ye, yr, fy[1]);
    dint_d2(yy2, ye, fy[2]);
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
    R[0] = R[0] / ex3;
    R[1] = R[1] / ex1;
    R[2] = R[2] / ex1;
    R[3] = R[3] / ex2;
    R[4] = R[4] / ex1;
    R[5] = R[5] / ex2;
}

// W layout: [6][lags][NLAM] (weight type major), already scaled by lambda and masked
__global__ void __launch_bounds__(256, 2) k_weights(const VbtTab *__restrict__ T, int Nx, int Ny, double dx, double dy,
                                                 double *W)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *g = reinterpret_cast<double2 *>(smem_raw);  // [VN][6]
    // [NLAM][6] weights at the top of g: the normalisation reads only g[NFIRST*6 .. (NLAST+1)*6), below it
    static_assert((NLAST + 1) * 6 * sizeof(double2) <= VN * 6 * sizeof(double2) - NLAM * 6 * sizeof(double),
                  "weights would overlap the samples still being read");
    double *wt = reinterpret_cast<double *>(smem_raw + VN * 6 * sizeof(double2) - NLAM * 6 * sizeof(double));
    __shared__ double w0[6], red[8][6];
    const int lag = blockIdx.x, lx = lag / Ny, ly = lag - lx * Ny;
    const size_t nlags = (size_t)Nx * Ny;
    // COMPUTE_WEIGHTS (calc_ie_tensor_module.F90:308-326) + VBTransformWeightsAllDoubleInt (:159-197)
    const double x = lx * dx + dx / 2.0, y = ly * dy + dy / 2.0;
    const double rho = sqrt(x * x + y * y);
    const double rp[6] = {rho * rho * rho, rho, rho, rho * rho, rho, rho * rho};
    const double alpha = dx / rho, beta = dy / rho, phi = atan2(y, x);
    const double cphi = cos(phi), sphi = sin(phi), s_arg = log(rho) - T->lambda_shift;
    for (int i = threadIdx.x; i < VN; i += blockDim.x) {
        double R[6];
        outfunc(i, s_arg, cphi, sphi, alpha, beta, R);
        const double sg = (i & 1) ? -1.0 : 1.0;
        const int p = T->inds[i];
        for (int c = 0; c < 6; c++) g[p * 6 + c] = make_double2(sg * R[c], 0.0);
    }
    __syncthreads();
    vbt_weights22(g, T);
    // normalisation (:282-285), real part for k in [NFIRST, NLAST], /hx/hy*rp, IE_* column order
    const int colmap[6] = {IE_D0, IE_DXX, IE_DXY, IE_DX, IE_DYY, IE_DY};  // COMPUTE_WEIGHTS :320-325
    for (int k = threadIdx.x; k < NLAM; k += blockDim.x) {
        const int idx = k + NFIRST;
        const double sg = (idx & 1) ? -1.0 : 1.0;
        for (int c = 0; c < 6; c++) {
            const double v = sg * g[idx * 6 + c].x / (double)VN;
            wt[k * 6 + colmap[c]] = v / dx / dy * rp[c];
        }
    }
    __syncthreads();
    // zeroing and maxima (:327-351)
    const bool lx0 = lx == 0, ly0 = ly == 0;
    for (int k = threadIdx.x; k < NLAM; k += blockDim.x) {
        if (lx0 || ly0) wt[k * 6 + IE_DXY] = 0.0;
        if (lx0) wt[k * 6 + IE_DX] = 0.0;
        if (ly0) wt[k * 6 + IE_DY] = 0.0;
    }
    __syncthreads();
    double mx[6] = {0, 0, 0, 0, 0, 0};
    for (int k = threadIdx.x; k < NLAM; k += blockDim.x)
        for (int c = 0; c < 6; c++) mx[c] = fmax(mx[c], fabs(wt[k * 6 + c]));
    for (int c = 0; c < 6; c++)
        for (int o = 16; o > 0; o >>= 1) mx[c] = fmax(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
    if ((threadIdx.x & 31) == 0)
        for (int c = 0; c < 6; c++) red[threadIdx.x >> 5][c] = mx[c];
    __syncthreads();
    if (threadIdx.x == 0) {
        double m[6] = {0, 0, 0, 0, 0, 0};
        for (int w = 0; w < (int)(blockDim.x >> 5); w++)
            for (int c = 0; c < 6; c++) m[c] = fmax(m[c], red[w][c]);
        w0[IE_DXX] = m[IE_DXX];
        if (!lx0 && !ly0) {
            const double mm = fmax(fmax(m[IE_DXY], m[IE_DYY]), fmax(m[IE_DX], m[IE_DY]));
            w0[IE_DXY] = w0[IE_DYY] = w0[IE_DX] = w0[IE_DY] = mm;
        } else if (lx0) {
            w0[IE_DXY] = -w0[IE_DXX];
            w0[IE_DYY] = m[IE_DYY];
            w0[IE_DX] = -w0[IE_DXX];
            w0[IE_DY] = ly0 ? -w0[IE_DXX] : m[IE_DY];
        } else {
            w0[IE_DXY] = -w0[IE_DXX];
            w0[IE_DYY] = m[IE_DYY];
            w0[IE_DX] = m[IE_DX];
            w0[IE_DY] = -w0[IE_DXX];
        }
        w0[IE_D0] = m[IE_D0];
    }
    __syncthreads();
    // threshold (:265-267) and lambda scalings (:268-274)
    for (int k = threadIdx.x; k < NLAM; k += blockDim.x) {
        double mxr = 0.0;
        for (int c = 0; c < 6; c++) mxr = fmax(mxr, fabs(wt[k * 6 + c] / w0[c]));
        const bool keep = mxr > WT_THRESHOLD;
        const double lm = T->lms[k];
        double v[6];
        v[IE_DXX] = wt[k * 6 + IE_DXX] / lm;
        v[IE_DYY] = wt[k * 6 + IE_DYY] / lm;
        v[IE_DXY] = wt[k * 6 + IE_DXY] / lm;
        v[IE_DX] = wt[k * 6 + IE_DX] * lm;
        v[IE_DY] = wt[k * 6 + IE_DY] * lm;
        v[IE_D0] = wt[k * 6 + IE_D0] * lm;
        for (int c = 0; c < 6; c++) W[((size_t)c * nlags + lag) * NLAM + k] = keep ? v[c] : 0.0;
    }
}

}  // namespace

int ie_green_tensor(IeOp *op, cudaStream_t st)
{
    const int Nx = op->Nx, Ny = op->Ny, Nz = op->Nz, Nl = op->Nl;
    if (Nl < 1 || Nl > MAXL || Nz > MAXZ) {
        g2_set_error_msg("Green's tensor on the GPU supports up to 16 layers and Nz <= 64");
        return G2_ERR_UNSUPPORTED;
    }
    const int P = op->P(), T = op->Tunit();
    const size_t lags = op->units();
    Bkg h{};
    h.Nl = Nl;
    h.Nz = Nz;
    const double mu0 = 4.0 * PI_D * 1e-7;
    for (int i = 0; i <= Nl; i++) {
        h.csigma[i] = op->csigma[i];
        // giem2g_interfaces.F90:278 k2 = i * csigma * mu0 * omega
        h.k2[i] = make_double2(-op->csigma[i].y * mu0 * op->omega, op->csigma[i].x * mu0 * op->omega);
    }
    for (int i = 1; i <= Nl - 1; i++) h.thick[i] = op->thick[i - 1];
    if (Nl > 1) {
        h.depth[1] = h.thick[1];
        for (int i = 2; i <= Nl - 1; i++) h.depth[i] = h.depth[i - 1] + h.thick[i];
    }
    h.iwm = make_double2(0.0, mu0 * op->omega);
    for (int i = 0; i <= Nz; i++) {
        h.L[i] = op->Lnumber[i];
        h.z[i] = op->z[i];
    }
    for (int i = 1; i <= Nz; i++) h.dz[i] = op->z[i] - op->z[i - 1];
    VbtTab *tab = new VbtTab();
    make_vbt(std::sqrt(op->dx * op->dx + op->dy * op->dy) / 2.0, *tab);  // calc_ie_tensor_module.F90:102-103

    Bkg *d_bkg = nullptr;
    VbtTab *d_tab = nullptr;
    double2 *M[4] = {nullptr, nullptr, nullptr, nullptr};
    double *W = nullptr;
    int rc = G2_OK;
    auto cleanup = [&]() {
        cudaFree(d_bkg);
        cudaFree(d_tab);
        for (auto p : M) cudaFree(p);
        cudaFree(W);
        delete tab;
    };
#define G2_TRY(expr)                                                      \
    do {                                                                  \
        cudaError_t e_ = (expr);                                          \
        if (e_ != cudaSuccess) {                                          \
            g2_set_error(__FILE__, __LINE__, cudaGetErrorString(e_));     \
            cleanup();                                                    \
            return G2_ERR_CUDA;                                           \
        }                                                                 \
    } while (0)
    G2_TRY(cudaMalloc(&d_bkg, sizeof(Bkg)));
    G2_TRY(cudaMalloc(&d_tab, sizeof(VbtTab)));
    G2_TRY(cudaMemcpyAsync(d_bkg, &h, sizeof(Bkg), cudaMemcpyHostToDevice, st));
    G2_TRY(cudaMemcpyAsync(d_tab, tab, sizeof(VbtTab), cudaMemcpyHostToDevice, st));
    G2_TRY(cudaMalloc(&M[0], sizeof(double2) * NLAM * P));
    G2_TRY(cudaMalloc(&M[1], sizeof(double2) * NLAM * P));
    G2_TRY(cudaMalloc(&M[2], sizeof(double2) * NLAM * Nz * Nz));
    G2_TRY(cudaMalloc(&M[3], sizeof(double2) * NLAM * P));
    G2_TRY(cudaMemsetAsync(M[2], 0, sizeof(double2) * NLAM * Nz * Nz, st));
    G2_TRY(cudaMalloc(&W, sizeof(double) * 6 * lags * NLAM));
    double *d_lms = reinterpret_cast<double *>(reinterpret_cast<char *>(d_tab) + offsetof(VbtTab, lms));
    k_basis<<<NLAM, 64, 0, st>>>(d_bkg, d_lms, M[0], M[1], M[2], M[3]);
    const size_t smw = sizeof(double2) * VN * 6;  // two blocks per SM
    G2_TRY(cudaFuncSetAttribute(k_weights, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smw));
    k_weights<<<(unsigned)lags, 256, smw, st>>>(d_tab, Nx, Ny, op->dx, op->dy, W);
    G2_TRY(cudaGetLastError());
    if (!op->d_spatial) G2_TRY(cudaMalloc(&op->d_spatial, lags * T * sizeof(double2)));
    const double sc = 1.0 / PI_D / 4.0;  // G1/PI/4 (calc_ie_tensor_module.F90:278-286)
    auto Wt = [&](int c) { return W + (size_t)c * lags * NLAM; };
    const int gm = (int)((lags + GM - 1) / GM);
    auto gemm = [&](const double *A1, const double2 *B1, const double *A2, const double2 *B2, int ncols, int off) {
        dim3 grid(gm, (ncols + GN - 1) / GN);
        k_gemm<<<grid, 256, 0, st>>>(A1, B1, A2, B2, (int)lags, ncols, op->d_spatial, T, off, sc);
    };
    gemm(Wt(IE_D0), M[0], Wt(IE_DXX), M[1], P, 0 * P);              // xx
    gemm(Wt(IE_DXY), M[1], nullptr, nullptr, P, 1 * P);             // xy
    gemm(Wt(IE_D0), M[0], Wt(IE_DYY), M[1], P, 2 * P);              // yy
    gemm(Wt(IE_D0), M[3], nullptr, nullptr, P, 3 * P);              // zz
    gemm(Wt(IE_DX), M[2], nullptr, nullptr, Nz * Nz, 4 * P);        // xz
    gemm(Wt(IE_DY), M[2], nullptr, nullptr, Nz * Nz, 4 * P + Nz * Nz);  // yz
    G2_TRY(cudaGetLastError());
    G2_TRY(cudaStreamSynchronize(st));
    cleanup();
#undef G2_TRY
    return rc;
}
