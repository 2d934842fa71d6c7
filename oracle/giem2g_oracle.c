/*
 * giem2g_oracle.c -- CPU FP64 restatement of GIEM2G's IE-solve path.
 *
 * TEST INFRASTRUCTURE ONLY: the correctness oracle for the B200 kernels.  The
 * product library never links or calls this code.  See giem2g_oracle.h for
 * layouts and the parity status (unpinned against reference outputs: the
 * reference has no tests and cannot be built here).
 *
 * Each routine cites the reference routine it restates (paths relative to the
 * GIEM2G source tree).  Array indices that the reference writes 1-based are
 * kept 1-based in local arrays where that makes the restatement easier to check.
 */
#include "giem2g_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_D 3.14159265358979323846264338327950288
/* const_module.F90:31-35 */
static double mu0_val(void) { return 4.0 * PI_D * 1e-7; }
static double eps0_val(void) { return 1.0 / (mu0_val() * 299792458.0 * 299792458.0); }
double orc_mu0(void) { return mu0_val(); }
double orc_eps0(void) { return eps0_val(); }
#define AIR_CONDUCTIVITY 1e-12

/* ------------------------------------------------------------------------- */
/* Layers: data_types_module.F90:214-242 (GetLayerSingle)                    */
/* depth is 1-based: depth[1..Nl-1]                                           */
/* ------------------------------------------------------------------------- */
int orc_get_layer(double z, int Nl, const double *depth)
{
    if (fabs(z) < 1e-15) return 0;
    if (z < 0) return -1;
    if (Nl == 1) return 1;
    int l = 1;
    if (z > depth[Nl - 1]) return Nl;
    while (z > depth[l]) l++;
    return l;
}

static void make_depth(const orc_model *m, double *depth /* Nl */)
{
    /* mpi_saveload_module.F90:57-60, giem2g_interfaces.F90:264-268 */
    depth[0] = 0.0;
    if (m->Nl > 1) {
        depth[1] = m->thick[0];
        for (int i = 2; i <= m->Nl - 1; i++) depth[i] = depth[i - 1] + m->thick[i - 1];
    }
}

/* giem2g_interfaces.F90:163-165 / mpi_saveload_module.F90:99-100 */
void orc_layer_numbers(const orc_model *m, int *L)
{
    double *depth = (double *)malloc(sizeof(double) * (m->Nl + 1));
    make_depth(m, depth);
    for (int i = 1; i <= m->Nz; i++) L[i] = orc_get_layer((m->z[i - 1] + m->z[i]) / 2.0, m->Nl, depth);
    L[0] = orc_get_layer(m->z[0] * (1.0 - 1e-7), m->Nl, depth);
    free(depth);
}

/* calc_ie_tensor_module.F90:295-306 (PreparePreconditioner) */
void orc_background_cells(const orc_model *m, double complex *csigb, double *sqsigb)
{
    int *L = (int *)malloc(sizeof(int) * (m->Nz + 1));
    orc_layer_numbers(m, L);
    for (int iz = 1; iz <= m->Nz; iz++) {
        csigb[iz - 1] = m->csigma[L[iz]];
        sqsigb[iz - 1] = sqrt(creal(m->csigma[L[iz]]));
    }
    free(L);
}

/* data_types_module.F90:244-259 (SET_FREQ) */
void orc_set_freq(int Nl, const double *sigma, double freq, int disp, double complex *csigma)
{
    double omega = freq * 2.0 * PI_D;
    if (disp) {
        csigma[0] = AIR_CONDUCTIVITY - I * omega * eps0_val();
        for (int i = 1; i <= Nl; i++) csigma[i] = sigma[i - 1] - I * omega * eps0_val();
    } else {
        csigma[0] = 0.0;
        for (int i = 1; i <= Nl; i++) csigma[i] = sigma[i - 1];
    }
}

/* ie_solver_module.F90:116-139 (SetAnomalySigma): file order (Nz,Nx,Ny) -> (Nx,Ny,Nz) */
void orc_set_anomaly_sigma(int Nx, int Ny, int Nz, const double *siga, double freq, int disp,
                           double complex *csiga)
{
    double w = freq * PI_D * 2.0;
    for (int iz = 0; iz < Nz; iz++)
        for (int iy = 0; iy < Ny; iy++)
            for (int ix = 0; ix < Nx; ix++) {
                double s = siga[((size_t)iy * Nx + ix) * Nz + iz];
                csiga[((size_t)iz * Ny + iy) * Nx + ix] = disp ? (s - I * w * eps0_val()) : s;
            }
}

/* ------------------------------------------------------------------------- */
/* Volume Bessel transform weights: VolumeBesselTransforms.F90 (FP64 branch)  */
/* ------------------------------------------------------------------------- */
#define VBT_N 1024
#define VBT_LOG2N 10
#define NFIRST 212 /* IntegralCodes.f90:2 */
#define NLAST 712  /* IntegralCodes.f90:3 */
#define NLAM (NLAST - NFIRST + 1)

static const double Y_STEP = 1e-1 * 2e0;                                      /* :41 */
static const double XI = -4.82205425726955430357775925664462079e-2 * 2e0;     /* :42 */
#define VBT_Q (Y_STEP / 2.0)                                                  /* :43 */
#define VBT_P (VBT_Q + XI)                                                    /* :44 */
#define VBT_N2 (-VBT_N / 2)                                                   /* :40 */

typedef struct {
    int inds[VBT_N];
    double complex w_fwd[VBT_N], w_bwd[VBT_N];
    double complex f1[VBT_N];
    double lms[NLAM];
    double lambda_shift;
} vbt_tables;

/* :620-629 bit_reverse: composition of circular right shifts of the low J bits */
static int vbt_bit_reverse(int i)
{
    int t = i;
    for (int J = VBT_LOG2N; J >= 2; J--) {
        int mask = (1 << J) - 1;
        int low = t & mask;
        low = (low >> 1) | ((low & 1) << (J - 1));
        t = (t & ~mask) | low;
    }
    return t;
}

/* :292-300 */
static double vbt_input_function(double t)
{
    double y = exp(-t);
    double y2 = y * y;
    double y4 = y2 * y2;
    return 8.0 * exp(-y2) * (y4 - 4.0 * y2 + 2.0) * y;
}

/* :630-649 FFT_16 (input in bit-reversed order), applied to `ncol` interleaved columns (:650-670) */
static void vbt_fft(double complex *x, int ncol, const double complex *wp)
{
    int I2 = 0;
    int J2 = 1;
    for (int i = 0; i < VBT_LOG2N; i++) {
        int Lstep = 2 * J2;
        for (int J = 0; J < J2; J++) {
            for (int Ip = J; Ip < VBT_N; Ip += Lstep) {
                int Iq = Ip + J2;
                for (int c = 0; c < ncol; c++) {
                    double complex temp = wp[I2] * x[(size_t)Iq * ncol + c];
                    x[(size_t)Iq * ncol + c] = x[(size_t)Ip * ncol + c] - temp;
                    x[(size_t)Ip * ncol + c] = x[(size_t)Ip * ncol + c] + temp;
                }
            }
            I2++;
        }
        J2 = Lstep;
    }
}

/* :111-139 VBTransformInit */
static void vbt_init(double s, vbt_tables *t)
{
    for (int i = 0; i < VBT_N; i++) t->inds[i] = vbt_bit_reverse(i);
    int I2 = 0;
    for (int i = 0; i < VBT_LOG2N; i++) {
        int K = 1 << i;
        for (int J = 0; J < K; J++) {
            double theta = -PI_D / K * J;
            t->w_fwd[I2] = cos(theta) + I * sin(theta);
            t->w_bwd[I2] = conj(t->w_fwd[I2]);
            I2++;
        }
    }
    for (int J = NFIRST; J <= NLAST; J++) t->lms[J - NFIRST] = exp(XI + (J + VBT_N2) * Y_STEP) / s;
    t->lambda_shift = log(s);
    for (int i = 0; i < VBT_N; i += 2) {
        double y1 = (i + VBT_N2) * Y_STEP + VBT_Q;
        t->f1[t->inds[i]] = vbt_input_function(y1);
        y1 = y1 + Y_STEP;
        t->f1[t->inds[i + 1]] = -vbt_input_function(y1);
    }
    vbt_fft(t->f1, 1, t->w_fwd);
}

typedef struct {
    double explt[VBT_N], explt2[VBT_N], explt3[VBT_N];
    double xy[2][VBT_N][3], xy2[2][VBT_N][3], xy_exp2[2][VBT_N][3], xy_erf[2][VBT_N][3];
} vbt_edt;

/* :142-157 CALC_EXP_LT */
static void vbt_calc_exp_lt(double s, vbt_edt *e)
{
    for (int i = 0; i < VBT_N; i += 2) {
        double y2 = (i + VBT_N2) * Y_STEP + VBT_P + s;
        e->explt[i] = exp(y2);
        e->explt2[i] = e->explt[i] * e->explt[i];
        e->explt3[i] = e->explt2[i] * e->explt[i];
        y2 = y2 + Y_STEP;
        e->explt[i + 1] = exp(y2);
        e->explt2[i + 1] = e->explt[i + 1] * e->explt[i + 1];
        e->explt3[i + 1] = e->explt2[i + 1] * e->explt[i + 1];
    }
}

/* :304-340 PrepareExps4 */
static void vbt_prepare_exps4(double phi, double alpha, double beta, vbt_edt *e)
{
    double cphi = cos(phi), sphi = sin(phi);
    for (int i = 0; i < VBT_N; i++) {
        double x1 = e->explt[i] * cphi;
        double y1 = e->explt[i] * sphi;
        double dxv = alpha * e->explt[i];
        double dyv = beta * e->explt[i];
        x1 = x1 - dxv * 0.5;
        y1 = y1 - dyv * 0.5;
        double x[3] = {x1, x1 + dxv, x1 - dxv};
        double y[3] = {y1, y1 + dyv, y1 - dyv};
        for (int k = 0; k < 3; k++) {
            x[k] = x[k] * 0.5;
            double x2 = x[k] * x[k];
            e->xy_exp2[0][i][k] = exp(-x2);
            e->xy_erf[0][i][k] = erf(x[k]);
            e->xy[0][i][k] = x[k];
            e->xy2[0][i][k] = x2;
            y[k] = y[k] * 0.5;
            double y2 = y[k] * y[k];
            e->xy_exp2[1][i][k] = exp(-y2);
            e->xy_erf[1][i][k] = erf(y[k]);
            e->xy[1][i][k] = y[k];
            e->xy2[1][i][k] = y2;
        }
    }
}

#define SPI_D 1.77245385090551602729816748334114518 /* sqrt(pi), :36 */
/* index helper: f(1..3) in the reference == f[0..2] here */
static void vbt_int_2d(const vbt_edt *e, int i, int j, double R[3]) /* :533-550 */
{
    const double *x = e->xy[j][i], *x2 = e->xy2[j][i], *ex = e->xy_exp2[j][i], *er = e->xy_erf[j][i];
    double f[3];
    for (int k = 0; k < 3; k++) f[k] = x[k] * er[k];
    R[0] = f[1] + f[2] - 2.0 * f[0];
    R[0] = R[0] * SPI_D * 0.25;
    for (int k = 0; k < 3; k++) f[k] = ex[k];
    R[1] = f[1] + f[2] - 2.0 * f[0];
    for (int k = 0; k < 3; k++) f[k] = ex[k] * x2[k] / 4.0;
    R[2] = f[1] + f[2] - 2.0 * f[0];
}
static void vbt_double_int_d0(const vbt_edt *e, int i, int j, double R[3]) /* :509-518 */
{
    double f[3];
    vbt_int_2d(e, i, j, f);
    R[0] = 32.0 * (1.5 * f[0] + f[1] + f[2]);
    R[1] = 8.0 * f[0] + 4.0 * f[1];
    R[2] = 4.0 * f[0] + f[1];
}
static void vbt_int_1d(const vbt_edt *e, int i, int j, double R[3]) /* :493-508 */
{
    const double *x = e->xy[j][i], *x2 = e->xy2[j][i], *ex = e->xy_exp2[j][i], *er = e->xy_erf[j][i];
    double f[3];
    for (int k = 0; k < 3; k++) f[k] = er[k];
    R[0] = f[1] + f[2] - 2.0 * f[0];
    R[0] = R[0] * SPI_D * 0.5;
    for (int k = 0; k < 3; k++) f[k] = ex[k] * x[k];
    R[1] = f[1] + f[2] - 2.0 * f[0];
    for (int k = 0; k < 3; k++) f[k] = f[k] * x2[k];
    R[2] = f[1] + f[2] - 2.0 * f[0];
}
static void vbt_double_int_d1(const vbt_edt *e, int i, int j, double R[3]) /* :470-480 */
{
    double f[3];
    vbt_int_1d(e, i, j, f);
    R[0] = -8.0 * f[2] - 12.0 * f[1] + 12.0 * f[0];
    R[1] = -2.0 * f[1] + 2.0 * f[0];
    R[2] = f[0];
}
static void vbt_double_int_d2(const vbt_edt *e, int i, int j, double R[3]) /* :437-452 */
{
    const double *x2 = e->xy2[j][i], *exv = e->xy_exp2[j][i];
    double ex[3], f[3];
    for (int k = 0; k < 3; k++) ex[k] = exv[k] / 2.0;
    for (int k = 0; k < 3; k++) f[k] = x2[k] * ex[k] * 4.0;
    R[1] = f[1] + f[2] - 2.0 * f[0];
    for (int k = 0; k < 3; k++) f[k] = x2[k] * f[k] * 4.0;
    R[0] = f[1] + f[2] - 2.0 * f[0];
    for (int k = 0; k < 3; k++) f[k] = ex[k];
    R[2] = f[1] + f[2] - 2.0 * f[0];
}

/* :377-403 outfunc_int4_all */
static void vbt_out_int4(const vbt_edt *e, int i, double R[6])
{
    double fx[3][3], fy[3][3]; /* [D][k] with D0=0,D1=1,D2=2 */
    vbt_double_int_d0(e, i, 0, fx[0]);
    vbt_double_int_d1(e, i, 0, fx[1]);
    vbt_double_int_d2(e, i, 0, fx[2]);
    vbt_double_int_d0(e, i, 1, fy[0]);
    vbt_double_int_d1(e, i, 1, fy[1]);
    vbt_double_int_d2(e, i, 1, fy[2]);
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
    R[0] = R[0] / e->explt3[i];
    R[1] = R[1] / e->explt[i];
    R[2] = R[2] / e->explt[i];
    R[3] = R[3] / e->explt2[i];
    R[4] = R[4] / e->explt[i];
    R[5] = R[5] / e->explt2[i];
}

/* :264-288 CalcWeights22 (non-Ooura branch) with the output function `outf`. WT[k][6] for k = NFIRST..NLAST */
typedef void (*vbt_outfunc)(const vbt_edt *e, int i, double R[6]);
static void vbt_calc_weights22_f(const vbt_tables *t, const vbt_edt *e, double *WT, vbt_outfunc outf)
{
    double complex *g = (double complex *)malloc(sizeof(double complex) * VBT_N * 6);
    double complex *h = (double complex *)malloc(sizeof(double complex) * VBT_N * 6);
    double R[6];
    for (int i = 0; i < VBT_N; i += 2) {
        outf(e, i, R);
        for (int c = 0; c < 6; c++) g[(size_t)t->inds[i] * 6 + c] = R[c];
        outf(e, i + 1, R);
        for (int c = 0; c < 6; c++) g[(size_t)t->inds[i + 1] * 6 + c] = -R[c];
    }
    vbt_fft(g, 6, t->w_fwd);
    for (int j = 0; j < VBT_N; j += 2)
        for (int c = 0; c < 6; c++) {
            h[(size_t)t->inds[j] * 6 + c] = g[(size_t)j * 6 + c] / t->f1[j];
            h[(size_t)t->inds[j + 1] * 6 + c] = -g[(size_t)(j + 1) * 6 + c] / t->f1[j + 1];
        }
    vbt_fft(h, 6, t->w_bwd);
    for (int j = 1; j < VBT_N; j += 2)
        for (int c = 0; c < 6; c++) {
            h[(size_t)(j - 1) * 6 + c] = h[(size_t)(j - 1) * 6 + c] / (double)VBT_N;
            h[(size_t)j * 6 + c] = -h[(size_t)j * 6 + c] / (double)VBT_N;
        }
    for (int k = NFIRST; k <= NLAST; k++)
        for (int c = 0; c < 6; c++) WT[(size_t)(k - NFIRST) * 6 + c] = creal(h[(size_t)k * 6 + c]);
    free(g);
    free(h);
}

static void vbt_calc_weights22(const vbt_tables *t, const vbt_edt *e, double *WT)
{
    vbt_calc_weights22_f(t, e, WT, vbt_out_int4);
}

/* :159-197 VBTransformWeightsAllDoubleInt */
static void vbt_weights_double_int(const vbt_tables *t, double x, double y, double hx, double hy, double *WT)
{
    double rho = sqrt(x * x + y * y);
    double rp[6] = {rho * rho * rho, rho, rho, rho * rho, rho, rho * rho};
    double alpha = hx / rho, beta = hy / rho, phi = atan2(y, x);
    vbt_edt *e = (vbt_edt *)malloc(sizeof(vbt_edt));
    vbt_calc_exp_lt(log(rho) - t->lambda_shift, e);
    vbt_prepare_exps4(phi, alpha, beta, e);
    vbt_calc_weights22(t, e, WT);
    for (int k = 0; k < NLAM; k++)
        for (int c = 0; c < 6; c++) WT[k * 6 + c] = WT[k * 6 + c] / hx / hy * rp[c];
    free(e);
}

int orc_vbt_weights(double x, double y, double hx, double hy, double rmin, double *WT, double *lms)
{
    vbt_tables *t = (vbt_tables *)malloc(sizeof(vbt_tables));
    vbt_init(rmin, t);
    vbt_weights_double_int(t, x, y, hx, hy, WT);
    if (lms) memcpy(lms, t->lms, sizeof(double) * NLAM);
    free(t);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Layered-medium recursions: apq_module.F90                                  */
/* Layer-indexed arrays are 1-based here: eta[1..Nl], p[l][2], ...            */
/* ------------------------------------------------------------------------- */
typedef struct {
    int Nl;
    const double complex *csigma; /* 0..Nl */
    double complex *k2;           /* 0..Nl */
    const double *thick;          /* thick[1..Nl-1] (shifted pointer) */
    double *depth;                /* depth[1..Nl-1] */
    double complex iwm;
} bkg_t;

/* apq_module.F90:267-290 Calc_p */
static void calc_p(const bkg_t *b, const double complex *eta, const double complex *el, double lms,
                   double complex (*p)[2])
{
    double complex eta0 = csqrt(lms * lms - b->k2[0]);
    double complex ceta = eta0 / eta[1];
    p[1][0] = (1.0 - ceta) / (1.0 + ceta);
    double complex cgamma = b->csigma[0] / b->csigma[1];
    p[1][1] = (cgamma - ceta) / (cgamma + ceta);
    for (int i = 2; i <= b->Nl; i++) {
        double complex w[2], a[2];
        w[0] = el[i - 1] * p[i - 1][0];
        w[1] = el[i - 1] * p[i - 1][1];
        for (int k = 0; k < 2; k++) w[k] = (w[k] - 1.0) / (w[k] + 1.0);
        a[0] = eta[i - 1] / eta[i];
        a[1] = a[0] * b->csigma[i] / b->csigma[i - 1];
        for (int k = 0; k < 2; k++) {
            w[k] = w[k] * a[k];
            p[i][k] = (1.0 + w[k]) / (1.0 - w[k]);
        }
    }
}

/* apq_module.F90:291-312 Calc_q */
static void calc_q(const bkg_t *b, const double complex *eta, const double complex *el, double complex (*q)[2])
{
    int Nl = b->Nl;
    q[Nl][0] = q[Nl][1] = 0.0;
    if (Nl > 1) {
        double complex a[2], w[2];
        a[0] = eta[Nl] / eta[Nl - 1];
        a[1] = a[0] * b->csigma[Nl - 1] / b->csigma[Nl];
        for (int k = 0; k < 2; k++) q[Nl - 1][k] = (1.0 - a[k]) / (1.0 + a[k]);
        for (int i = Nl - 2; i >= 1; i--) {
            w[0] = el[i + 1] * q[i + 1][0];
            w[1] = el[i + 1] * q[i + 1][1];
            for (int k = 0; k < 2; k++) w[k] = (w[k] - 1.0) / (w[k] + 1.0);
            a[0] = eta[i + 1] / eta[i];
            a[1] = a[0] * b->csigma[i] / b->csigma[i + 1];
            for (int k = 0; k < 2; k++) {
                w[k] = w[k] * a[k];
                q[i][k] = (1.0 + w[k]) / (1.0 - w[k]);
            }
        }
    }
}

/* apq_module.F90:230-266 Calc_Apq.  A (optional) is [Nl+1][Nl+1][2], 1-based */
static void calc_apq(const bkg_t *b, double lms, double complex (*Arr)[2], double complex (*p)[2],
                     double complex (*q)[2], double complex *eta, double complex *A)
{
    int Nl = b->Nl;
    double complex el[Nl + 1];
    for (int i = 1; i <= Nl; i++) eta[i] = csqrt(lms * lms - b->k2[i]);
    for (int i = 1; i <= Nl - 1; i++) el[i] = cexp(-2.0 * eta[i] * b->thick[i]);
    el[Nl] = 0.0;
    calc_p(b, eta, el, lms, p);
    calc_q(b, eta, el, q);
    for (int i = 1; i <= Nl; i++)
        for (int k = 0; k < 2; k++) Arr[i][k] = 1.0 / eta[i] / (1.0 - p[i][k] * q[i][k] * el[i]);
    if (A) {
#define AIX(i, j, k) A[(((size_t)(i) * (Nl + 1)) + (j)) * 2 + (k)]
        double complex w[Nl + 1][2];
        for (int i = 1; i <= Nl - 1; i++) {
            double complex tmp = (b->k2[i] - b->k2[i + 1]);
            tmp = b->depth[i] * tmp;
            tmp = tmp / (eta[i + 1] + eta[i]);
            for (int k = 0; k < 2; k++) w[i][k] = (1.0 + p[i + 1][k]) / (1.0 + p[i][k] * el[i]) * cexp(tmp);
        }
        for (int i = 1; i <= Nl; i++) {
            AIX(i, i, 0) = Arr[i][0];
            AIX(i, i, 1) = Arr[i][1];
            for (int j = i - 1; j >= 1; j--) {
                for (int k = 0; k < 2; k++) AIX(j, i, k) = AIX(j + 1, i, k) * w[j][k];
                AIX(i, j, 0) = AIX(j, i, 0);
                AIX(i, j, 1) = AIX(j, i, 1) * b->csigma[i] / b->csigma[j];
            }
        }
#undef AIX
    }
}

typedef struct {
    int Nz;
    const int *L;        /* Lnumber[0..Nz] */
    const double *z;     /* z[0..Nz] */
    const double *dz;    /* dz[1..Nz] (shifted) */
} anom_t;

/* apq_module.F90:112-137 Calc_pexpz_All */
static void calc_pexpz(const bkg_t *b, const anom_t *a, const double complex *expz, const double complex *eta,
                       double complex (*p)[2], double complex (*pexpz)[2])
{
    int l = a->L[0];
    double complex e;
    if (l > 1) e = cexp(-2.0 * eta[l] * (a->z[0] - b->depth[l - 1]));
    else if (l == 1) e = cexp(-2.0 * eta[1] * (a->z[0]));
    else e = 1.0;
    for (int i = 1; i <= a->Nz; i++) {
        if (l != a->L[i]) e = 1.0;
        l = a->L[i];
        pexpz[i][0] = e * p[l][0];
        pexpz[i][1] = e * p[l][1];
        e = e * expz[i] * expz[i];
    }
}

/* apq_module.F90:155-177 Calc_qexpz_All */
static void calc_qexpz(const bkg_t *b, const anom_t *a, const double complex *expz, const double complex *eta,
                       double complex (*q)[2], double complex (*qexpz)[2])
{
    int l = a->L[a->Nz];
    double complex e;
    if (l != b->Nl) e = cexp(-2.0 * eta[l] * (b->depth[l] - a->z[a->Nz]));
    else e = 0.0;
    for (int i = a->Nz; i >= 1; i--) {
        if (l != a->L[i]) e = 1.0;
        l = a->L[i];
        qexpz[i][0] = e * q[l][0];
        qexpz[i][1] = e * q[l][1];
        e = e * expz[i] * expz[i];
    }
}

/* apq_module.F90:83-110 Calc_tframe_p */
static void calc_tframe(const bkg_t *b, const anom_t *an, const double complex *expz, const double complex *eta,
                        double complex (*pexpz)[2], double complex (*fcont)[2], double complex (*tframe)[3])
{
    for (int i = 1; i <= an->Nz - 1; i++) {
        int l = an->L[i];
        double complex a[2], bb[2], c[2];
        for (int k = 0; k < 2; k++) {
            a[k] = pexpz[i][k];
            bb[k] = a[k] * expz[i];
            c[k] = bb[k] * expz[i];
            a[k] = 1.0 + a[k];
            bb[k] = 1.0 + bb[k];
            c[k] = 1.0 + c[k];
        }
        double complex w = (1.0 - expz[i]) / eta[l];
        for (int k = 0; k < 2; k++) fcont[i][k] = expz[i] * a[k] / c[k];
        tframe[i][0] = w * bb[0] / c[0];
        tframe[i][1] = 1.0 - fcont[i][1];
        tframe[i][2] = w * bb[1] / c[1];
        tframe[i][1] = tframe[i][1] / b->csigma[l];
        tframe[i][2] = tframe[i][2] / b->csigma[l];
    }
}

/* apq_module.F90:138-153 Calc_bframe_q */
static void calc_bframe(const bkg_t *b, const anom_t *an, const double complex *expz,
                        double complex (*qexpz)[2], double complex *fcont, double complex *bframe)
{
    for (int i = an->Nz; i >= 2; i--) {
        int l = an->L[i];
        double complex a = qexpz[i][1];
        double complex d = 1.0 + a * expz[i] * expz[i];
        a = 1.0 + a;
        fcont[i] = expz[i] * a / d;
        bframe[i] = (fcont[i] - 1.0) / b->csigma[l];
    }
}

/* apq_module.F90:31-79 Calc_FtFb */
static void calc_ftfb(const bkg_t *b, const anom_t *an, const double complex *expz, double complex (*pexpz)[2],
                      double complex (*qexpz)[2], const double complex *eta, double complex (*Arr)[2],
                      double complex (*Ft)[3], double complex *Fb, double complex (*GII)[4])
{
    for (int i = 1; i <= an->Nz; i++) {
        int l = an->L[i];
        double complex a[2], a1[2], a2[2], p1[2], p2[2], pe1[2], pe2[2], q1[2], q2[2], qe1[2], qe2[2], w[2], Fb3[3];
        for (int k = 0; k < 2; k++) {
            a[k] = (1.0 - expz[i]) * Arr[l][k];
            a1[k] = a[k] / eta[l];
            a2[k] = a1[k] / eta[l];
            p1[k] = 1.0 + pexpz[i][k];
            p2[k] = 1.0 - pexpz[i][k];
            pe1[k] = 1.0 + pexpz[i][k] * expz[i];
            pe2[k] = -1.0 + pexpz[i][k] * expz[i];
            q1[k] = 1.0 + qexpz[i][k];
            q2[k] = 1.0 - qexpz[i][k];
            qe1[k] = 1.0 + qexpz[i][k] * expz[i];
            qe2[k] = 1.0 - qexpz[i][k] * expz[i];
        }
        double complex eta2 = eta[l] * eta[l];
        for (int k = 0; k < 2; k++) Ft[i][k] = a1[k] * p1[k] * qe1[k];
        Ft[i][2] = a[1] * p1[1] * qe2[1];
        for (int k = 0; k < 2; k++) Fb3[k] = a1[k] * pe1[k] * q1[k];
        Fb3[2] = a[1] * pe2[1] * q1[1];
        for (int k = 0; k < 2; k++) w[k] = -a2[k] * (p2[k] * qe1[k] + pe1[k] * q2[k]);
        double dzi = an->dz[i];
        GII[i][0] = w[0] + 2.0 / eta2 * dzi;
        GII[i][1] = Fb3[1] - Ft[i][1];
        GII[i][2] = (w[1] + 2.0 / eta2 * dzi) * b->iwm + eta2 / b->csigma[l] * w[1];
        GII[i][3] = Fb3[2] - Ft[i][2] - eta2 * w[0];
        Fb[i] = Fb3[1];
    }
}

/* IE_DXX.. ie_kernel_hankel_module.F90:29-35 (0-based here) */
enum { IE_DXX = 0, IE_DXY = 1, IE_DYY = 2, IE_DX = 3, IE_DY = 4, IE_D0 = 5 };
/* EXX.. const_module.F90:100-108 (0-based here) */
enum { G_EXX = 0, G_EXY = 1, G_EXZ = 2, G_EYY = 3, G_EYZ = 4, G_EZZ = 5 };
#define G1IX(c, r, s) (((size_t)(c) * Nz + ((r)-1)) * Nz + ((s)-1)) /* G(c, Izr, Izs) 1-based rows */

/* ie_kernel_hankel_module.F90:125-173 GoByShellsU */
static void go_by_shells_u(int Izs, int Nz, double lms2, const double complex *fb, double complex (*fcont)[2],
                           double complex (*frame)[3], const double *WT, double complex iwm, double complex *G)
{
    double complex f1wdxx = fb[0] * (WT[IE_DXX] + WT[IE_D0]) * iwm;
    double complex f1wdyy = fb[0] * (WT[IE_DYY] + WT[IE_D0]) * iwm;
    double complex f1wdxy = fb[0] * WT[IE_DXY] * iwm;
    double complex f2wdx = fb[1] * WT[IE_DX];
    double complex f2wdy = fb[1] * WT[IE_DY];
    double complex f2wdzz = fb[1] * WT[IE_D0] * lms2;
    double complex f3wdxx = fb[2] * WT[IE_DXX];
    double complex f3wdyy = fb[2] * WT[IE_DYY];
    double complex f3wdxy = fb[2] * WT[IE_DXY];
    for (int r = Izs - 1; r >= 1; r--) {
        G[G1IX(G_EXX, r, Izs)] = f1wdxx * frame[r][0] + f3wdxx * frame[r][1] + G[G1IX(G_EXX, r, Izs)];
        G[G1IX(G_EXY, r, Izs)] = f3wdxy * frame[r][1] + f1wdxy * frame[r][0] + G[G1IX(G_EXY, r, Izs)];
        G[G1IX(G_EXZ, r, Izs)] = f2wdx * frame[r][1] + G[G1IX(G_EXZ, r, Izs)];
        G[G1IX(G_EYY, r, Izs)] = f1wdyy * frame[r][0] + f3wdyy * frame[r][1] + G[G1IX(G_EYY, r, Izs)];
        G[G1IX(G_EYZ, r, Izs)] = f2wdy * frame[r][1] + G[G1IX(G_EYZ, r, Izs)];
        G[G1IX(G_EZZ, r, Izs)] = f2wdzz * frame[r][2] + G[G1IX(G_EZZ, r, Izs)];
        f1wdxx = f1wdxx * fcont[r][0];
        f1wdyy = f1wdyy * fcont[r][0];
        f1wdxy = f1wdxy * fcont[r][0];
        f2wdx = f2wdx * fcont[r][1];
        f2wdy = f2wdy * fcont[r][1];
        f2wdzz = f2wdzz * fcont[r][1];
        f3wdxx = f3wdxx * fcont[r][1];
        f3wdyy = f3wdyy * fcont[r][1];
        f3wdxy = f3wdxy * fcont[r][1];
    }
}

/* ie_kernel_hankel_module.F90:175-197 GoByShellsL */
static void go_by_shells_l(int Izs, int Nz, double complex fb, const double complex *fcont,
                           const double complex *frame, const double *WT, double complex *G)
{
    double complex f2wdx = fb * WT[IE_DX];
    double complex f2wdy = fb * WT[IE_DY];
    for (int r = Izs + 1; r <= Nz; r++) {
        G[G1IX(G_EXZ, r, Izs)] = f2wdx * frame[r] + G[G1IX(G_EXZ, r, Izs)];
        G[G1IX(G_EYZ, r, Izs)] = f2wdy * frame[r] + G[G1IX(G_EYZ, r, Izs)];
        f2wdx = f2wdx * fcont[r];
        f2wdy = f2wdy * fcont[r];
    }
}

/* ie_kernel_hankel_module.F90:44-122 Calc_Double_Integral_U */
static void calc_double_integral_u(const bkg_t *b, const anom_t *an, double lms, const double *WT,
                                   double complex *G)
{
    int Nl = b->Nl, Nz = an->Nz;
    double complex p[Nl + 1][2], q[Nl + 1][2], eta[Nl + 1], Arr[Nl + 1][2];
    double complex expz[Nz + 1], pez[Nz + 1][2], qez[Nz + 1][2], fcont_t[Nz + 1][2], tframe[Nz + 1][3];
    double complex fcont_b[Nz + 1], bframe[Nz + 1], Ft[Nz + 1][3], Fb[Nz + 1], GII[Nz + 1][4];
    calc_apq(b, lms, Arr, p, q, eta, NULL);
    for (int iz = 1; iz <= Nz; iz++) expz[iz] = cexp(-eta[an->L[iz]] * (an->dz[iz]));
    calc_pexpz(b, an, expz, eta, p, pez);
    calc_tframe(b, an, expz, eta, pez, fcont_t, tframe);
    calc_qexpz(b, an, expz, eta, q, qez);
    calc_bframe(b, an, expz, qez, fcont_b, bframe);
    calc_ftfb(b, an, expz, pez, qez, eta, Arr, Ft, Fb, GII);
    double lm2 = lms * lms;
    for (int iz = 1; iz <= Nz; iz++) {
        int l = an->L[iz];
        double complex f1wdxx = GII[iz][0] * WT[IE_DXX] * lm2;
        double complex f1wdyy = GII[iz][0] * WT[IE_DYY] * lm2;
        double complex f1wdxy = GII[iz][0] * WT[IE_DXY] * lm2;
        double complex f2wdx = GII[iz][1] * WT[IE_DX];
        double complex f2wdy = GII[iz][1] * WT[IE_DY];
        double complex f2wdzz = (GII[iz][2]) * WT[IE_D0];
        double complex f3wdxx = GII[iz][3] * WT[IE_DXX];
        double complex f3wdyy = GII[iz][3] * WT[IE_DYY];
        double complex f3wdxy = GII[iz][3] * WT[IE_DXY];
        double complex cs = b->csigma[l];
        G[G1IX(G_EXX, iz, iz)] = (GII[iz][0] * WT[IE_D0] * b->iwm + (f1wdxx + f3wdxx) / cs) + G[G1IX(G_EXX, iz, iz)];
        G[G1IX(G_EXY, iz, iz)] = (f1wdxy + f3wdxy) / cs + G[G1IX(G_EXY, iz, iz)];
        G[G1IX(G_EXZ, iz, iz)] = f2wdx / cs + G[G1IX(G_EXZ, iz, iz)];
        G[G1IX(G_EYY, iz, iz)] = (GII[iz][0] * WT[IE_D0] * b->iwm + (f1wdyy + f3wdyy) / cs) + G[G1IX(G_EYY, iz, iz)];
        G[G1IX(G_EYZ, iz, iz)] = f2wdy / cs + G[G1IX(G_EYZ, iz, iz)];
        G[G1IX(G_EZZ, iz, iz)] = f2wdzz + G[G1IX(G_EZZ, iz, iz)];
        go_by_shells_u(iz, Nz, lm2, Ft[iz], fcont_t, tframe, WT, b->iwm, G);
        go_by_shells_l(iz, Nz, Fb[iz], fcont_b, bframe, WT, G);
    }
}

static void make_bkg(const orc_model *m, bkg_t *b, double *depth_store, double complex *k2_store)
{
    b->Nl = m->Nl;
    b->csigma = m->csigma;
    make_depth(m, depth_store);
    b->depth = depth_store;
    b->thick = m->thick - 1; /* thick[1..Nl-1] */
    /* giem2g_interfaces.F90:277-280 CREATE_BACKGROUND */
    for (int i = 0; i <= m->Nl; i++) k2_store[i] = I * m->csigma[i] * mu0_val() * m->omega;
    b->k2 = k2_store;
    b->iwm = I * mu0_val() * m->omega;
}

/* calc_ie_tensor_module.F90:308-352 COMPUTE_WEIGHTS */
static void compute_weights(const vbt_tables *t, int lx, int ly, double dx, double dy, double *WT, double *W0)
{
    double *WT0 = (double *)malloc(sizeof(double) * NLAM * 6);
    double x = lx * dx + dx / 2.0;
    double y = ly * dy + dy / 2.0;
    vbt_weights_double_int(t, x, y, dx, dy, WT0);
    for (int k = 0; k < NLAM; k++) {
        WT[k * 6 + IE_D0] = WT0[k * 6 + 0];
        WT[k * 6 + IE_DXX] = WT0[k * 6 + 1];
        WT[k * 6 + IE_DXY] = WT0[k * 6 + 2];
        WT[k * 6 + IE_DX] = WT0[k * 6 + 3];
        WT[k * 6 + IE_DYY] = WT0[k * 6 + 4];
        WT[k * 6 + IE_DY] = WT0[k * 6 + 5];
    }
    free(WT0);
#define COLMAX(c) ({ double mm_ = 0; for (int k_ = 0; k_ < NLAM; k_++) { double a_ = fabs(WT[k_ * 6 + (c)]); if (a_ > mm_) mm_ = a_; } mm_; })
#define COLZERO(c) do { for (int k_ = 0; k_ < NLAM; k_++) WT[k_ * 6 + (c)] = 0.0; } while (0)
    W0[IE_DXX] = COLMAX(IE_DXX);
    if (lx != 0 && ly != 0) {
        double mm = 0;
        for (int c = IE_DXY; c <= IE_DY; c++) { double v = COLMAX(c); if (v > mm) mm = v; }
        for (int c = IE_DXY; c <= IE_DY; c++) W0[c] = mm;
    } else if (lx == 0) {
        COLZERO(IE_DXY);
        W0[IE_DXY] = -W0[IE_DXX];
        W0[IE_DYY] = COLMAX(IE_DYY);
        COLZERO(IE_DX);
        W0[IE_DX] = -W0[IE_DXX];
        if (ly != 0) {
            W0[IE_DY] = COLMAX(IE_DY);
        } else {
            COLZERO(IE_DY);
            W0[IE_DY] = -W0[IE_DXX];
        }
    } else {
        COLZERO(IE_DXY);
        W0[IE_DXY] = -W0[IE_DXX];
        W0[IE_DYY] = COLMAX(IE_DYY);
        W0[IE_DX] = COLMAX(IE_DX);
        COLZERO(IE_DY);
        W0[IE_DY] = -W0[IE_DXX];
    }
    W0[IE_D0] = COLMAX(IE_D0);
#undef COLMAX
#undef COLZERO
}

#define WT_THRESHOLD 1e-12 /* calc_ie_tensor_module.F90:37 */

/* calc_ie_tensor_module.F90:241-293 CalcIntegralGreenTensor3dElementGeneral */
static void green_element(const vbt_tables *t, const bkg_t *b, const anom_t *an, int lx, int ly, double dx,
                          double dy, double complex *symm /* [4][P] */, double complex *asym /* [2][Nz*Nz] */)
{
    int Nz = an->Nz;
    double *WT = (double *)malloc(sizeof(double) * NLAM * 6);
    double W0[6], W[6];
    compute_weights(t, lx, ly, dx, dy, WT, W0);
    double complex *G = (double complex *)calloc((size_t)6 * Nz * Nz, sizeof(double complex));
    for (int k = 0; k < NLAM; k++) {
        double mx = 0;
        for (int c = 0; c < 6; c++) {
            double wm = fabs(WT[k * 6 + c] / W0[c]);
            if (wm > mx) mx = wm;
        }
        if (mx > WT_THRESHOLD) {
            double lm = t->lms[k];
            W[IE_DXX] = WT[k * 6 + IE_DXX] / lm;
            W[IE_DYY] = WT[k * 6 + IE_DYY] / lm;
            W[IE_DXY] = WT[k * 6 + IE_DXY] / lm;
            W[IE_DX] = WT[k * 6 + IE_DX] * lm;
            W[IE_DY] = WT[k * 6 + IE_DY] * lm;
            W[IE_D0] = WT[k * 6 + IE_D0] * lm;
            calc_double_integral_u(b, an, lm, W, G);
        }
    }
    int P = Nz * (Nz + 1) / 2;
    for (int s = 1; s <= Nz; s++)
        for (int r = 1; r <= Nz; r++) {
            /* G_asym(Izr, Izs) column-major, :278-279 */
            asym[0 * Nz * Nz + (s - 1) * Nz + (r - 1)] = G[G1IX(G_EXZ, r, s)] / PI_D / 4.0;
            asym[1 * Nz * Nz + (s - 1) * Nz + (r - 1)] = G[G1IX(G_EYZ, r, s)] / PI_D / 4.0;
        }
    for (int iz = 1; iz <= Nz; iz++)
        for (int iz0 = 1; iz0 <= iz; iz0++) {
            int idx = iz0 + iz * (iz - 1) / 2 - 1; /* :283-286 packed upper */
            symm[0 * P + idx] = G[G1IX(G_EXX, iz0, iz)] / PI_D / 4.0;
            symm[1 * P + idx] = G[G1IX(G_EXY, iz0, iz)] / PI_D / 4.0;
            symm[2 * P + idx] = G[G1IX(G_EYY, iz0, iz)] / PI_D / 4.0;
            symm[3 * P + idx] = G[G1IX(G_EZZ, iz0, iz)] / PI_D / 4.0;
        }
    free(G);
    free(WT);
}

/* calc_ie_tensor_module.F90:54-192 CalcIntegralGreenTensor, all lags of one process */
int orc_green_tensor(const orc_model *m, double complex *symm, double complex *asym, int nthreads)
{
    int Nx = m->Nx, Ny = m->Ny, Nz = m->Nz;
    int P = Nz * (Nz + 1) / 2;
    double *depth = (double *)malloc(sizeof(double) * (m->Nl + 1));
    double complex *k2 = (double complex *)malloc(sizeof(double complex) * (m->Nl + 1));
    bkg_t b;
    make_bkg(m, &b, depth, k2);
    int *L = (int *)malloc(sizeof(int) * (Nz + 1));
    orc_layer_numbers(m, L);
    double *dz = (double *)malloc(sizeof(double) * (Nz + 1));
    for (int i = 1; i <= Nz; i++) dz[i] = m->z[i] - m->z[i - 1];
    anom_t an = {Nz, L, m->z, dz};
    vbt_tables *t = (vbt_tables *)malloc(sizeof(vbt_tables));
    double rmin = sqrt(m->dx * m->dx + m->dy * m->dy) / 2.0; /* :102 */
    vbt_init(rmin, t);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
#endif
    for (int lx = 0; lx < Nx; lx++)
        for (int ly = 0; ly < Ny; ly++) {
            size_t u = (size_t)lx * Ny + ly;
            green_element(t, &b, &an, lx, ly, m->dx, m->dy, symm + u * 4 * P, asym + u * 2 * Nz * Nz);
        }
    free(t);
    free(dz);
    free(L);
    free(k2);
    free(depth);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* FFT helpers (the reference calls FFTW; this is a plain radix-2 / DFT)      */
/* sign = -1 forward (FFTW_FORWARD), +1 backward, unnormalised                */
/* ------------------------------------------------------------------------- */
static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void fft1d(double complex *x, int n, int stride, int sign, double complex *work)
{
    for (int i = 0; i < n; i++) work[i] = x[(size_t)i * stride];
    if (is_pow2(n)) {
        /* bit reversal */
        for (int i = 1, j = 0; i < n; i++) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) { double complex t = work[i]; work[i] = work[j]; work[j] = t; }
        }
        for (int len = 2; len <= n; len <<= 1) {
            for (int k = 0; k < len / 2; k++) {
                double ang = sign * 2.0 * PI_D * k / len;
                double complex w = cos(ang) + I * sin(ang);
                for (int i = 0; i < n; i += len) {
                    double complex u = work[i + k], v = work[i + k + len / 2] * w;
                    work[i + k] = u + v;
                    work[i + k + len / 2] = u - v;
                }
            }
        }
        for (int i = 0; i < n; i++) x[(size_t)i * stride] = work[i];
    } else {
        for (int k = 0; k < n; k++) {
            double complex s = 0;
            for (int j = 0; j < n; j++) {
                double ang = sign * 2.0 * PI_D * (double)(((long)j * k) % n) / n;
                s += work[j] * (cos(ang) + I * sin(ang));
            }
            x[(size_t)k * stride] = s;
        }
    }
}

/* 2-D DFT of a (n2 rows) x (n1 cols) plane, row-major [i2][i1] */
static void fft2d(double complex *a, int n1, int n2, int sign, double complex *work)
{
    for (int i2 = 0; i2 < n2; i2++) fft1d(a + (size_t)i2 * n1, n1, 1, sign, work);
    for (int i1 = 0; i1 < n1; i1++) fft1d(a + i1, n2, n1, sign, work);
}

/* ------------------------------------------------------------------------- */
/* Tensor spectrum: Integral_Equation_Module.F90:319-471 with                 */
/* Distributed_FFT.F90:507-551 (y mirror + Nyquist), restated for one process */
/* Parities (sx,sy): xx(+,+) xy(-,-) yy(+,+) zz(+,+) xz(-,+) yz(+,-)  :334-346 */
/* The x-Nyquist correction uses s = (-1)^kx (the sign `ss` at :396/:419/:461 */
/* is only initialised for odd NxHalf in the reference; this is the intended  */
/* value, which makes the apply an exact block-Toeplitz product).             */
/* ------------------------------------------------------------------------- */
static void spectrum_component(int Nx, int Ny, const double complex *src, size_t src_stride, size_t n_elem,
                               double sx, double sy, double complex *dst, size_t dst_stride, int nthreads)
{
    int n1 = 2 * Nx, n2 = 2 * Ny;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
        double complex *plane = (double complex *)malloc(sizeof(double complex) * n1 * n2);
        double complex *work = (double complex *)malloc(sizeof(double complex) * (n1 > n2 ? n1 : n2));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
        for (size_t e = 0; e < n_elem; e++) {
            memset(plane, 0, sizeof(double complex) * n1 * n2);
            /* plane[ky-lag][kx-lag]; src indexed [lx][ly] */
            for (int lx = 0; lx < Nx; lx++)
                for (int ly = 0; ly < Ny; ly++) plane[(size_t)ly * n1 + lx] = src[((size_t)lx * Ny + ly) * src_stride + e];
            /* x mirror (Integral_Equation_Module.F90:441-447), lag Nx := 0 */
            for (int ly = 0; ly < Ny; ly++) {
                for (int ix = 1; ix <= Nx - 1; ix++) plane[(size_t)ly * n1 + (n1 - ix)] = sx * plane[(size_t)ly * n1 + ix];
                plane[(size_t)ly * n1 + Nx] = 0.0;
            }
            /* y mirror (Distributed_FFT.F90:530-536), lag Ny := 0 */
            for (int iy = 1; iy <= Ny - 1; iy++)
                for (int ix = 0; ix < n1; ix++) plane[(size_t)(n2 - iy) * n1 + ix] = sy * plane[(size_t)iy * n1 + ix];
            for (int ix = 0; ix < n1; ix++) plane[(size_t)Ny * n1 + ix] = 0.0;
            fft2d(plane, n1, n2, -1, work);
            /* y Nyquist correction (Distributed_FFT.F90:540-545) on all kx columns */
            for (int ix = 0; ix < n1; ix++) {
                double complex tmp = plane[(size_t)Ny * n1 + ix];
                double t = 1.0;
                for (int iy = 0; iy < n2; iy++) {
                    plane[(size_t)iy * n1 + ix] -= t * tmp;
                    t = -t;
                }
            }
            /* keep kx<Nx, ky<Ny, then x Nyquist correction (Integral_Equation_Module.F90:459-466) */
            for (int ky = 0; ky < Ny; ky++) {
                double complex tmp = plane[(size_t)ky * n1 + Nx];
                double s = 1.0;
                for (int kx = 0; kx < Nx; kx++) {
                    dst[((size_t)kx * Ny + ky) * dst_stride + e] = plane[(size_t)ky * n1 + kx] - tmp * s;
                    s = -s;
                }
            }
        }
        free(work);
        free(plane);
    }
}

int orc_tensor_spectrum(int Nx, int Ny, int Nz, const double complex *symm, const double complex *asym,
                        double complex *symm_hat, double complex *asym_hat, int nthreads)
{
    int P = Nz * (Nz + 1) / 2;
    const double ssx[4] = {1, -1, 1, 1}, ssy[4] = {1, -1, 1, 1};
    for (int c = 0; c < 4; c++)
        spectrum_component(Nx, Ny, symm + (size_t)c * P, (size_t)4 * P, P, ssx[c], ssy[c], symm_hat + (size_t)c * P,
                           (size_t)4 * P, nthreads);
    const double asx[2] = {-1, 1}, asy[2] = {1, -1};
    for (int c = 0; c < 2; c++)
        spectrum_component(Nx, Ny, asym + (size_t)c * Nz * Nz, (size_t)2 * Nz * Nz, (size_t)Nz * Nz, asx[c], asy[c],
                           asym_hat + (size_t)c * Nz * Nz, (size_t)2 * Nz * Nz, nthreads);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* BLAS level-2 semantics used by the contraction                             */
/* ------------------------------------------------------------------------- */
/* ZSPMV('U', n, alpha, AP, x, 1, beta, y, 1) */
static void zspmv_u(int n, double complex alpha, const double complex *ap, const double complex *x,
                    double complex beta, double complex *y)
{
    double complex t[n];
    for (int i = 0; i < n; i++) t[i] = 0;
    for (int j = 0; j < n; j++)
        for (int i = 0; i <= j; i++) {
            double complex a = ap[i + j * (j + 1) / 2];
            t[i] += a * x[j];
            if (i != j) t[j] += a * x[i];
        }
    for (int i = 0; i < n; i++) y[i] = (beta == 0 ? 0 : beta * y[i]) + alpha * t[i];
}
/* ZGEMV(trans, n, n, alpha, A(col-major), n, x, 1, beta, y, 1), trans 'N' or 'T' */
static void zgemv_sq(char trans, int n, double complex alpha, const double complex *A, const double complex *x,
                     double complex beta, double complex *y)
{
    double complex t[n];
    for (int i = 0; i < n; i++) t[i] = 0;
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            if (trans == 'N') t[i] += A[i + (size_t)j * n] * x[j];
            else t[j] += A[i + (size_t)j * n] * x[i];
        }
    for (int i = 0; i < n; i++) y[i] = (beta == 0 ? 0 : beta * y[i]) + alpha * t[i];
}

/* apply_ie_operator_module.F90:265-296 / :298-327, one spectral point.
 * u/w: [3][Nz] (component x,y,z).  sx = +1 slot1 (kx>=0), -1 slot2; m = MirrorY */
static void vertical_mult(int Nz, const double complex *gs /*[4][P]*/, const double complex *ga /*[2][Nz*Nz]*/,
                          double sxv, double m, const double complex *u, double complex *w)
{
    int P = Nz * (Nz + 1) / 2;
    const double complex *ux = u, *uy = u + Nz, *uz = u + 2 * Nz;
    double complex *wx = w, *wy = w + Nz, *wz = w + 2 * Nz;
    zspmv_u(Nz, 1.0, gs + 0 * P, ux, 0.0, wx);
    zspmv_u(Nz, sxv * m, gs + 1 * P, uy, 1.0, wx);
    zspmv_u(Nz, sxv * m, gs + 1 * P, ux, 0.0, wy);
    zspmv_u(Nz, 1.0, gs + 2 * P, uy, 1.0, wy);
    zspmv_u(Nz, 1.0, gs + 3 * P, uz, 0.0, wz);
    zgemv_sq('N', Nz, sxv, ga + 0, uz, 1.0, wx);
    zgemv_sq('T', Nz, -sxv, ga + 0, ux, 1.0, wz);
    zgemv_sq('N', Nz, m, ga + (size_t)Nz * Nz, uz, 1.0, wy);
    zgemv_sq('T', Nz, -m, ga + (size_t)Nz * Nz, uy, 1.0, wz);
}

/* APPLY_PRECOND (apply_ie_operator_module.F90:39-178) + MULT_IE_OP (:189-263) for one process holding all rows */
int orc_apply(int Nx, int Ny, int Nz, const double complex *symm_hat, const double complex *asym_hat,
              const double complex *csiga, const double complex *csigb, const double *sqsigb, const double *dz,
              const double complex *v_in, double complex *v_out, int nthreads)
{
    int n1 = 2 * Nx, n2 = 2 * Ny, P = Nz * (Nz + 1) / 2;
    size_t plane = (size_t)n1 * n2, cells = (size_t)Nx * Ny * Nz;
    double complex *buf = (double complex *)calloc(plane * 3 * Nz, sizeof(double complex));
    double complex *out = (double complex *)calloc(plane * 3 * Nz, sizeof(double complex));
    /* pre-step :57-114 */
    for (int c = 0; c < 3; c++)
        for (int iz = 0; iz < Nz; iz++)
            for (int iy = 0; iy < Ny; iy++)
                for (int ix = 0; ix < Nx; ix++) {
                    size_t cell = ((size_t)iz * Ny + iy) * Nx + ix;
                    double complex asiga = 2.0 * sqsigb[iz] / (csiga[cell] + conj(csigb[iz]));
                    double complex dsig = csiga[cell] - csigb[iz];
                    double complex gsig = dsig * asiga;
                    buf[((size_t)c * Nz + iz) * plane + (size_t)iy * n1 + ix] = v_in[c * cells + cell] * gsig;
                }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
    {
        double complex *work = (double complex *)malloc(sizeof(double complex) * (n1 > n2 ? n1 : n2));
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int pl = 0; pl < 3 * Nz; pl++) fft2d(buf + (size_t)pl * plane, n1, n2, -1, work);
        /* contraction :230-248 -- every (kx,ky) except the Nyquist row/column */
        double complex u[3 * Nz], w[3 * Nz];
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int q = 0; q < Nx; q++) {
            for (int r = 0; r < Ny; r++) {
                const double complex *gs = symm_hat + ((size_t)q * Ny + r) * 4 * P;
                const double complex *ga = asym_hat + ((size_t)q * Ny + r) * 2 * Nz * Nz;
                for (int slot = 0; slot < 2; slot++) {
                    if (slot == 1 && q == 0) continue; /* kx=0 has one slot; slot 2 there is the Nyquist */
                    int kx = slot == 0 ? q : n1 - q;
                    for (int mir = 0; mir < 2; mir++) {
                        if (mir == 1 && r == 0) continue; /* duplicate ky=0 row is discarded */
                        int ky = mir == 0 ? r : n2 - r;
                        size_t off = (size_t)ky * n1 + kx;
                        for (int k = 0; k < 3 * Nz; k++) u[k] = buf[(size_t)k * plane + off];
                        vertical_mult(Nz, gs, ga, slot == 0 ? 1.0 : -1.0, mir == 0 ? 1.0 : -1.0, u, w);
                        for (int k = 0; k < 3 * Nz; k++) out[(size_t)k * plane + off] = w[k];
                    }
                }
            }
        }
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int pl = 0; pl < 3 * Nz; pl++) fft2d(out + (size_t)pl * plane, n1, n2, +1, work);
        free(work);
    }
    /* post-step :125-174 */
    double N = 4.0 * Nx * Ny;
    for (int c = 0; c < 3; c++)
        for (int iz = 0; iz < Nz; iz++)
            for (int iy = 0; iy < Ny; iy++)
                for (int ix = 0; ix < Nx; ix++) {
                    size_t cell = ((size_t)iz * Ny + iy) * Nx + ix;
                    double complex asiga = 2.0 * sqsigb[iz] / (csiga[cell] + conj(csigb[iz]));
                    double complex d1 = v_in[c * cells + cell] * asiga;
                    double complex d2 = d1 - out[((size_t)c * Nz + iz) * plane + (size_t)iy * n1 + ix] / (dz[iz]) / N;
                    v_out[c * cells + cell] = d2 * sqsigb[iz];
                }
    free(out);
    free(buf);
    return 0;
}

/* Dense block-Toeplitz brute force.  Kernel for lag (lx,ly), |lx|<Nx, |ly|<Ny:
 * g_c extended by the component parities; zx(z,z') = -xz(z',z), zy(z,z') = -yz(z',z). */
int orc_apply_toeplitz(int Nx, int Ny, int Nz, const double complex *symm, const double complex *asym,
                       const double complex *csiga, const double complex *csigb, const double *sqsigb,
                       const double *dz, const double complex *v_in, double complex *v_out)
{
    int P = Nz * (Nz + 1) / 2;
    size_t cells = (size_t)Nx * Ny * Nz;
    double complex *u = (double complex *)malloc(sizeof(double complex) * 3 * cells);
    double complex *w = (double complex *)calloc(3 * cells, sizeof(double complex));
    for (int iz = 0; iz < Nz; iz++)
        for (int iy = 0; iy < Ny; iy++)
            for (int ix = 0; ix < Nx; ix++) {
                size_t cell = ((size_t)iz * Ny + iy) * Nx + ix;
                double complex asiga = 2.0 * sqsigb[iz] / (csiga[cell] + conj(csigb[iz]));
                double complex gsig = (csiga[cell] - csigb[iz]) * asiga;
                for (int c = 0; c < 3; c++) u[c * cells + cell] = v_in[c * cells + cell] * gsig;
            }
#define SY(a, b) ((a) <= (b) ? (a) + (b) * ((b) + 1) / 2 : (b) + (a) * ((a) + 1) / 2)
    for (int y = 0; y < Ny; y++)
        for (int x = 0; x < Nx; x++)
            for (int yp = 0; yp < Ny; yp++)
                for (int xp = 0; xp < Nx; xp++) {
                    int lx = x - xp, ly = y - yp;
                    int ax = lx < 0 ? -lx : lx, ay = ly < 0 ? -ly : ly;
                    double nx = lx < 0 ? -1.0 : 1.0, ny = ly < 0 ? -1.0 : 1.0;
                    size_t unit = (size_t)ax * Ny + ay;
                    const double complex *gs = symm + unit * 4 * P;
                    const double complex *ga = asym + unit * 2 * Nz * Nz;
                    for (int z = 0; z < Nz; z++) {
                        size_t co = ((size_t)z * Ny + y) * Nx + x;
                        double complex sx_ = 0, sy_ = 0, sz_ = 0;
                        for (int zp = 0; zp < Nz; zp++) {
                            size_t ci = ((size_t)zp * Ny + yp) * Nx + xp;
                            double complex ux = u[ci], uy = u[cells + ci], uz = u[2 * cells + ci];
                            double complex gxx = gs[0 * P + SY(z, zp)], gxy = nx * ny * gs[1 * P + SY(z, zp)];
                            double complex gyy = gs[2 * P + SY(z, zp)], gzz = gs[3 * P + SY(z, zp)];
                            double complex gxz = nx * ga[(size_t)zp * Nz + z];          /* xz(z,z') */
                            double complex gzx = -nx * ga[(size_t)z * Nz + zp];         /* -xz(z',z) */
                            double complex gyz = ny * ga[(size_t)Nz * Nz + (size_t)zp * Nz + z];
                            double complex gzy = -ny * ga[(size_t)Nz * Nz + (size_t)z * Nz + zp];
                            sx_ += gxx * ux + gxy * uy + gxz * uz;
                            sy_ += gxy * ux + gyy * uy + gyz * uz;
                            sz_ += gzx * ux + gzy * uy + gzz * uz;
                        }
                        w[co] += sx_;
                        w[cells + co] += sy_;
                        w[2 * cells + co] += sz_;
                    }
                }
#undef SY
    for (int iz = 0; iz < Nz; iz++)
        for (int iy = 0; iy < Ny; iy++)
            for (int ix = 0; ix < Nx; ix++) {
                size_t cell = ((size_t)iz * Ny + iy) * Nx + ix;
                double complex asiga = 2.0 * sqsigb[iz] / (csiga[cell] + conj(csigb[iz]));
                for (int c = 0; c < 3; c++)
                    v_out[c * cells + cell] = (v_in[c * cells + cell] * asiga - w[c * cells + cell] / dz[iz]) * sqsigb[iz];
            }
    free(w);
    free(u);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Plane wave RHS: sources_module.F90:67-101 (PlaneWaveIntegral)              */
/* ------------------------------------------------------------------------- */
int orc_plane_wave(const orc_model *m, int pol, double complex *E0)
{
    int Nl = m->Nl, Nx = m->Nx, Ny = m->Ny, Nz = m->Nz;
    double depth[Nl + 1];
    double complex k2[Nl + 1];
    bkg_t b;
    make_bkg(m, &b, depth, k2);
    double complex Arr[Nl + 1][2], p[Nl + 1][2], q[Nl + 1][2], eta[Nl + 1];
    double complex *A = (double complex *)calloc((size_t)(Nl + 1) * (Nl + 1) * 2, sizeof(double complex));
    calc_apq(&b, 0.0, Arr, p, q, eta, A);
#define AIX(i, j, k) A[(((size_t)(i) * (Nl + 1)) + (j)) * 2 + (k)]
    double complex t1;
    if (Nl > 1) t1 = 1.0 + q[1][0] * cexp(-b.depth[1] * eta[1] * 2.0);
    else t1 = 1.0;
    t1 = AIX(1, 1, 0) * t1;
    int L[Nz + 1];
    orc_layer_numbers(m, L);
    size_t cells = (size_t)Nx * Ny * Nz;
    memset(E0, 0, sizeof(double complex) * 3 * cells);
    for (int iz = 1; iz <= Nz; iz++) {
        double dzv = m->z[iz] - m->z[iz - 1];
        int l = L[iz];
        double complex e1 = cexp(-eta[l] * m->z[iz - 1]);
        double complex e2 = cexp(-eta[l] * m->z[iz]);
        double complex e3, e4;
        if (l < Nl) {
            e3 = q[l][0] * (cexp(-eta[l] * (2.0 * b.depth[l] - m->z[iz - 1])));
            e4 = q[l][0] * (cexp(-eta[l] * (2.0 * b.depth[l] - m->z[iz])));
        } else {
            e3 = e4 = 0.0;
        }
        double complex G = (e1 - e2 + e4 - e3) * AIX(l, 1, 0) / t1;
        G = G / dzv / eta[l];
        for (size_t k = 0; k < (size_t)Nx * Ny; k++) E0[(size_t)pol * cells + (size_t)(iz - 1) * Nx * Ny + k] = G;
    }
#undef AIX
    free(A);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Nested FGMRES: GFGMRES/gmres.F90 + seq_fgmres.F90, depth 2                */
/* ------------------------------------------------------------------------- */
typedef struct gm_ctx gm_ctx;
typedef void (*gm_apply_fn)(void *A, const double complex *in, double complex *out);
typedef struct gm_solver {
    int flex, n, m, maxit;
    double tol;
    double complex *x, *y, *r0, *w, *dots, *V, *H, *Z, *gsin;
    double *gcos;
    int iternum;
    gm_apply_fn apply;
    void *A;
    struct gm_solver *precond; /* inner solver used as right preconditioner */
    orc_result info;
    double *history;
    int history_len;
    int *apply_count;
} gm_solver;

#define ZERO_THRESHOLD 1e-14    /* gmres.F90:21 */
#define N_IGS_ITER 3            /* gmres.F90:22 */

static double complex zdotc(int n, const double complex *a, const double complex *b)
{
    double complex s = 0;
    for (int i = 0; i < n; i++) s += conj(a[i]) * b[i];
    return s;
}
static double vnorm(int n, const double complex *v) { return sqrt(creal(zdotc(n, v, v))); } /* gmres.F90:537-549 */

/* netlib ZROTG */
static void zrotg(double complex *ca, double complex cb, double *c, double complex *s)
{
    if (cabs(*ca) == 0.0) {
        *c = 0.0;
        *s = 1.0;
        *ca = cb;
    } else {
        double scale = cabs(*ca) + cabs(cb);
        double a1 = cabs(*ca / scale), b1 = cabs(cb / scale);
        double norm = scale * sqrt(a1 * a1 + b1 * b1);
        double complex alpha = *ca / cabs(*ca);
        *c = cabs(*ca) / norm;
        *s = alpha * conj(cb) / norm;
        *ca = alpha * norm;
    }
}
/* netlib ZROT (one element) */
static void zrot1(double complex *cx, double complex *cy, double c, double complex s)
{
    double complex t = c * *cx + s * *cy;
    *cy = c * *cy - conj(s) * *cx;
    *cx = t;
}

#define HIX(s, i, j) ((s)->H[((size_t)((j)-1)) * ((s)->m + 1) + ((i)-1)]) /* Hessenberg(i,j), 1-based, col-major */
#define VCOL(s, j) ((s)->V + (size_t)((j)-1) * (s)->n)
#define ZCOL(s, j) ((s)->Z + (size_t)((j)-1) * (s)->n)

static void gm_apply(gm_solver *s, const double complex *in, double complex *out)
{
    s->apply(s->A, in, out);
    if (s->apply_count) (*s->apply_count)++;
}
static void gmres_solve(gm_solver *s, double complex *x, const double complex *x0, const double complex *b,
                        orc_result *info);

/* gmres.F90:491-506 ApplyRightPreconditioner; seq_fgmres.F90:142-152 */
static void apply_right_precond(gm_solver *s, const double complex *vin, double complex *vout, int K)
{
    if (s->precond) {
        orc_result inf;
        gmres_solve(s->precond, vout, vin, vin, &inf);
    } else {
        memcpy(vout, vin, sizeof(double complex) * s->n);
    }
    if (s->flex) memcpy(ZCOL(s, K), vout, sizeof(double complex) * s->n);
}

/* gmres.F90:216-329 KrylovSubspaceConstruction */
static double krylov(gm_solver *s, double bn, int *jH)
{
    int N = s->n, M = s->m;
    double bea = -1.0;
    for (;;) {
        int j = *jH;
        apply_right_precond(s, VCOL(s, j), s->w, j);
        gm_apply(s, s->w, s->r0);
        memcpy(s->w, s->r0, sizeof(double complex) * N); /* ApplyLeftPreconditioner: copy */
        for (int i = 1; i <= j; i++) HIX(s, i, j) = 0;
        double dloo = 0, dnormw = 0;
        int northo = 0;
        for (;;) {
            northo++;
            for (int k = 1; k <= j; k++) s->dots[k - 1] = zdotc(N, VCOL(s, k), s->w);
            for (int k = 1; k <= j; k++) HIX(s, k, j) += s->dots[k - 1];
            for (int i = 0; i < N; i++) {
                double complex acc = 0;
                for (int k = 1; k <= j; k++) acc += VCOL(s, k)[i] * s->dots[k - 1];
                s->w[i] -= acc;
            }
            double d2 = 0;
            for (int k = 0; k < j; k++) d2 += creal(s->dots[k]) * creal(s->dots[k]) + cimag(s->dots[k]) * cimag(s->dots[k]);
            dloo = sqrt(d2);
            dnormw = vnorm(N, s->w);
            if ((2.0 * dnormw > dloo) || (northo > N_IGS_ITER)) break;
        }
        HIX(s, j + 1, j) = dnormw;
        for (int i = 0; i < N; i++) VCOL(s, j + 1)[i] = s->w[i] / dnormw;
        for (int i = 1; i <= j - 1; i++) zrot1(&HIX(s, i, j), &HIX(s, i + 1, j), s->gcos[i - 1], s->gsin[i - 1]);
        double complex h1 = HIX(s, j, j);
        zrotg(&h1, HIX(s, j + 1, j), &s->gcos[j - 1], &s->gsin[j - 1]);
        zrot1(&HIX(s, j, M + 1), &HIX(s, j + 1, M + 1), s->gcos[j - 1], s->gsin[j - 1]);
        zrot1(&HIX(s, j, j), &HIX(s, j + 1, j), s->gcos[j - 1], s->gsin[j - 1]);
        HIX(s, j + 1, j) = 0;
        double dnormres = cabs(HIX(s, j + 1, M + 1));
        bea = dnormres / bn;
        s->iternum++;
        if (s->history && s->iternum <= s->history_len) s->history[s->iternum - 1] = bea;
        (*jH)++;
        if (bea < s->tol || *jH > M) break;
    }
    return bea;
}

/* gmres.F90:423-485 ConstructCurrentSolution + projection */
static void construct_solution(gm_solver *s, int jH, double complex *sol)
{
    int N = s->n, M = s->m, L = jH - 1;
    for (int i = 1; i <= L; i++) s->y[i - 1] = HIX(s, i, M + 1);
    /* ZTRSV('U','N','N') */
    for (int i = L; i >= 1; i--) {
        double complex t = s->y[i - 1];
        for (int k = i + 1; k <= L; k++) t -= HIX(s, i, k) * s->y[k - 1];
        s->y[i - 1] = t / HIX(s, i, i);
    }
    for (int i = 0; i < N; i++) {
        double complex acc = 0;
        for (int k = 1; k <= L; k++) acc += (s->flex ? ZCOL(s, k)[i] : VCOL(s, k)[i]) * s->y[k - 1];
        s->x[i] = acc;
    }
    if (s->flex) memcpy(s->r0, s->x, sizeof(double complex) * N);
    else apply_right_precond(s, s->x, s->r0, L); /* no preconditioner on the inner level: copy */
    for (int i = 0; i < N; i++) {
        s->x[i] = s->r0[i] + sol[i];
        sol[i] = s->x[i];
    }
}

/* gmres.F90:382-421 FinalActions */
static double final_actions(gm_solver *s, int jH, double sPb, const double complex *rhs, double complex *sol)
{
    int N = s->n;
    construct_solution(s, jH, sol);
    memcpy(s->w, sol, sizeof(double complex) * N);
    gm_apply(s, s->w, s->r0);
    for (int i = 0; i < N; i++) {
        s->r0[i] = rhs[i] - s->r0[i];
        s->w[i] = s->r0[i];
    }
    double res = vnorm(N, s->w) / sPb;
    s->info.stat = res >= s->tol ? 2 : 1;
    return res;
}

/* gmres.F90:333-379 PrepareRestart, RESTART_RESIDUAL = .FALSE. branch */
static double prepare_restart(gm_solver *s, const double complex *rhs, double complex *sol, int jH)
{
    (void)rhs;
    int N = s->n, M = s->m;
    construct_solution(s, jH, sol);
    double beta = cabs(HIX(s, M + 1, M + 1));
    for (int j = M; j >= 1; j--) {
        HIX(s, j, M + 1) = 0;
        zrot1(&HIX(s, j, M + 1), &HIX(s, j + 1, M + 1), s->gcos[j - 1], -s->gsin[j - 1]);
    }
    for (int i = 0; i < N; i++) {
        double complex acc = 0;
        for (int k = 1; k <= M + 1; k++) acc += VCOL(s, k)[i] * HIX(s, k, M + 1);
        s->w[i] = acc;
    }
    return beta;
}

/* gmres.F90:110-213 GMRES_SOLVE */
static void gmres_solve(gm_solver *s, double complex *x, const double complex *x0, const double complex *b,
                        orc_result *info)
{
    int N = s->n, M = s->m;
    memset(s->H, 0, sizeof(double complex) * (M + 1) * (M + 1));
    s->iternum = 0;
    double be = -1, bea = -1;
    double bn = vnorm(N, b);
    if (bn < ZERO_THRESHOLD) {
        memset(x, 0, sizeof(double complex) * N);
        info->stat = 1;
        info->iterations = 0;
        return;
    }
    double sPb = bn, sb = bn;
    memcpy(x, x0, sizeof(double complex) * N);
    gm_apply(s, x0, s->r0);
    for (int i = 0; i < N; i++) s->r0[i] = b[i] - s->r0[i];
    memcpy(s->w, s->r0, sizeof(double complex) * N);
    double beta = vnorm(N, s->w);
    if (beta / sb < s->tol) {
        info->stat = 1;
        info->be = beta / sb;
        info->iterations = 0;
        return;
    }
    int iter = 0, jH = 1;
    for (;;) {
        HIX(s, 1, M + 1) = beta;
        for (int i = 0; i < N; i++) VCOL(s, 1)[i] = s->w[i] / beta;
        for (int i = 1; i <= M; i++) HIX(s, i + 1, M + 1) = 0;
        jH = 1;
        bea = krylov(s, bn, &jH);
        if (bea < s->tol) {
            be = final_actions(s, jH, sPb, b, x);
            info->stat = s->info.stat;
            info->iterations = s->iternum;
            info->be = be;
            info->bea = bea;
            return;
        }
        iter++;
        if (iter >= s->maxit) break;
        beta = prepare_restart(s, b, x, jH);
    }
    be = final_actions(s, jH, sPb, b, x);
    info->bea = bea;
    info->be = be;
    info->iterations = s->iternum;
    info->stat = -1;
}

static void gm_alloc(gm_solver *s, int n, int m, int flex)
{
    memset(s, 0, sizeof(*s));
    s->n = n;
    s->m = m;
    s->flex = flex;
    s->x = (double complex *)calloc(n, sizeof(double complex));
    s->y = (double complex *)calloc(m, sizeof(double complex));
    s->r0 = (double complex *)calloc(n, sizeof(double complex));
    s->w = (double complex *)calloc(n, sizeof(double complex));
    s->dots = (double complex *)calloc(m + 1, sizeof(double complex));
    s->V = (double complex *)calloc((size_t)n * (m + 1), sizeof(double complex));
    s->H = (double complex *)calloc((size_t)(m + 1) * (m + 1), sizeof(double complex));
    s->gsin = (double complex *)calloc(m, sizeof(double complex));
    s->gcos = (double *)calloc(m, sizeof(double));
    if (flex) s->Z = (double complex *)calloc((size_t)n * m, sizeof(double complex));
}
static void gm_free(gm_solver *s)
{
    free(s->x); free(s->y); free(s->r0); free(s->w); free(s->dots); free(s->V); free(s->H);
    free(s->gsin); free(s->gcos); free(s->Z);
}

typedef struct {
    int Nx, Ny, Nz, nthreads;
    const double complex *sh, *ah, *csiga, *csigb;
    const double *sqsigb, *dz;
} op_ctx;
static void op_apply(void *A, const double complex *in, double complex *out)
{
    op_ctx *o = (op_ctx *)A;
    orc_apply(o->Nx, o->Ny, o->Nz, o->sh, o->ah, o->csiga, o->csigb, o->sqsigb, o->dz, in, out, o->nthreads);
}

/* ie_solver_module.F90:43-114 SolveEquation + :141-258 GIEM2G_FGMRES (single process: no halving) */
int orc_solve(int Nx, int Ny, int Nz, const double complex *symm_hat, const double complex *asym_hat,
              const double complex *csiga, const double complex *csigb, const double *sqsigb, const double *dz,
              const double complex *E_bkg, const double complex *E0, int outer_buf, int inner_buf,
              int max_restart, double tol, double complex *Esol, orc_result *info, double *hist, int hist_len,
              int nthreads)
{
    size_t cells = (size_t)Nx * Ny * Nz;
    int N = (int)(3 * cells);
    op_ctx o = {Nx, Ny, Nz, nthreads, symm_hat, asym_hat, csiga, csigb, sqsigb, dz};
    double complex *rhs = (double complex *)malloc(sizeof(double complex) * N);
    double complex *guess = (double complex *)malloc(sizeof(double complex) * N);
    for (int c = 0; c < 3; c++)
        for (size_t cell = 0; cell < cells; cell++) {
            int iz = (int)(cell / ((size_t)Nx * Ny));
            rhs[c * cells + cell] = sqsigb[iz] * E_bkg[c * cells + cell];
        }
    if (E0) {
        for (int c = 0; c < 3; c++)
            for (size_t cell = 0; cell < cells; cell++) {
                int iz = (int)(cell / ((size_t)Nx * Ny));
                double complex asiga = 2.0 * sqsigb[iz] / (csiga[cell] + conj(csigb[iz]));
                guess[c * cells + cell] = E0[c * cells + cell] / asiga;
            }
    } else {
        memcpy(guess, rhs, sizeof(double complex) * N);
    }
    /* seq_fgmres.F90:35-67 INIT_SEQ_FGMRES depth 2 */
    gm_solver outer, inner;
    gm_alloc(&outer, N, outer_buf, 1);
    gm_alloc(&inner, N, inner_buf, 0);
    int applies = 0;
    inner.maxit = 1;
    inner.tol = tol;
    inner.apply = op_apply;
    inner.A = &o;
    inner.apply_count = &applies;
    outer.maxit = max_restart;
    outer.tol = tol;
    outer.apply = op_apply;
    outer.A = &o;
    outer.precond = &inner;
    outer.apply_count = &applies;
    outer.history = hist;
    outer.history_len = hist_len;
    orc_result r;
    memset(&r, 0, sizeof(r));
    gmres_solve(&outer, Esol, guess, rhs, &r);
    r.applies = applies;
    if (info) *info = r;
    /* :85-97 E := a * chi */
    for (int c = 0; c < 3; c++)
        for (size_t cell = 0; cell < cells; cell++) {
            int iz = (int)(cell / ((size_t)Nx * Ny));
            double complex asiga = 2.0 * sqsigb[iz] / (csiga[cell] + conj(csigb[iz]));
            Esol[c * cells + cell] = asiga * Esol[c * cells + cell];
        }
    gm_free(&outer);
    gm_free(&inner);
    free(rhs);
    free(guess);
    return 0;
}

/* ========================================================================= */
/* Receiver continuation (fields at receivers from the anomaly's currents)   */
/* Continuation_Function_Module.F90, calc_rc_tensor_module.F90,              */
/* rc_kernel_hankel_module.F90, VolumeBesselTransforms.F90 (single integral) */
/* ========================================================================= */

/* data_types_module.F90:124-152 PrepareRecvs: receiver layer and the number of anomaly cells above it;
 * a receiver strictly inside a cell is moved to the cell's top border. */
int orc_prepare_receivers(const orc_model *m, int Nr, double *zrecv, int *recv_layer, int *anom_cell)
{
    double depth[m->Nl + 1];
    make_depth(m, depth);
    int Nz = m->Nz;
    for (int i = 0; i < Nr; i++) {
        double zr = zrecv[i];
        int l = orc_get_layer(zr, m->Nl, depth);
        recv_layer[i] = l > 1 ? l : 1;
        if (zr <= m->z[0]) {
            anom_cell[i] = 0;
        } else if (zr >= m->z[Nz]) {
            anom_cell[i] = Nz + 1;
        } else {
            for (int iz = 1; iz <= Nz; iz++) {
                if (fabs(zr / m->z[iz] - 1.0) < 1e-7) {
                    anom_cell[i] = iz;
                    break;
                } else if (zr > m->z[iz - 1] && zr < m->z[iz]) {
                    zrecv[i] = m->z[iz - 1];
                    anom_cell[i] = iz - 1;
                    break;
                }
            }
        }
    }
    return 0;
}

/* VolumeBesselTransforms.F90:342-371 PrepareExps2 */
static void vbt_prepare_exps2(double phi, double alpha, double beta, vbt_edt *e)
{
    double cphi = cos(phi), sphi = sin(phi);
    for (int i = 0; i < VBT_N; i++) {
        double x1 = e->explt[i] * cphi * 0.5;
        double y1 = e->explt[i] * sphi * 0.5;
        double dxv = alpha * e->explt[i] * 0.5;
        double dyv = beta * e->explt[i] * 0.5;
        double x[2] = {x1, x1 + dxv}, y[2] = {y1, y1 + dyv};
        for (int k = 0; k < 2; k++) {
            double x2 = x[k] * x[k];
            e->xy_exp2[0][i][k] = exp(-x2);
            e->xy_erf[0][i][k] = erf(x[k]);
            e->xy[0][i][k] = x[k];
            e->xy2[0][i][k] = x2;
            double y2 = y[k] * y[k];
            e->xy_exp2[1][i][k] = exp(-y2);
            e->xy_erf[1][i][k] = erf(y[k]);
            e->xy[1][i][k] = y[k];
            e->xy2[1][i][k] = y2;
        }
    }
}

static void vbt_single_int_d0(const vbt_edt *e, int i, int j, double R[3]) /* :553-567 */
{
    const double *x = e->xy[j][i], *x2 = e->xy2[j][i], *ex = e->xy_exp2[j][i], *er = e->xy_erf[j][i];
    double f[2];
    for (int k = 0; k < 2; k++) f[k] = er[k] * SPI_D;
    double a = f[1] - f[0];
    R[0] = a * 0.5;
    for (int k = 0; k < 2; k++) f[k] = x[k] * ex[k];
    double b = f[1] - f[0];
    R[1] = a - 2.0 * b;
    for (int k = 0; k < 2; k++) f[k] = f[k] * x2[k];
    double c = f[1] - f[0];
    R[2] = 6.0 * a - 12.0 * b - 8.0 * c;
}
static void vbt_single_int_d1(const vbt_edt *e, int i, int j, double R[3]) /* :569-585 */
{
    const double *x2 = e->xy2[j][i], *ex = e->xy_exp2[j][i];
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
static void vbt_single_int_d2(const vbt_edt *e, int i, int j, double R[3]) /* :587-603 */
{
    const double *x = e->xy[j][i], *x2 = e->xy2[j][i], *ex = e->xy_exp2[j][i];
    double f[2];
    for (int k = 0; k < 2; k++) f[k] = x[k] * ex[k];
    double a = f[1] - f[0];
    R[0] = -a * 0.5;
    for (int k = 0; k < 2; k++) f[k] = f[k] * x2[k];
    double b = f[1] - f[0];
    R[1] = 2.0 * (a - b);
    for (int k = 0; k < 2; k++) f[k] = f[k] * x2[k];
    double c = f[1] - f[0];
    R[2] = 16.0 * b - 8.0 * c;
}

/* :407-434 outfunc_int2_all */
static void vbt_out_int2(const vbt_edt *e, int i, double R[6])
{
    double fx[3][3], fy[3][3];
    vbt_single_int_d0(e, i, 0, fx[0]);
    vbt_single_int_d1(e, i, 0, fx[1]);
    vbt_single_int_d2(e, i, 0, fx[2]);
    vbt_single_int_d0(e, i, 1, fy[0]);
    vbt_single_int_d1(e, i, 1, fy[1]);
    vbt_single_int_d2(e, i, 1, fy[2]);
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
    R[0] = R[0] / e->explt[i];
    R[1] = R[1] * e->explt[i];
    R[2] = R[2] * e->explt[i];
    R[4] = R[4] * e->explt[i];
}

/* :198-229 VBTransformWeightsAllSingleInt: WT[k][6] (columns in the routine's own order) */
static void vbt_weights_single_int(const vbt_tables *t, double x, double y, double hx, double hy, double *WT)
{
    double rho = sqrt(x * x + y * y);
    double alpha = hx / rho, beta = hy / rho, phi = atan2(y, x);
    vbt_edt *e = (vbt_edt *)malloc(sizeof(vbt_edt));
    vbt_calc_exp_lt(log(rho) - t->lambda_shift, e);
    vbt_prepare_exps2(phi, alpha, beta, e);
    vbt_calc_weights22_f(t, e, WT, vbt_out_int2);
    for (int k = 0; k < NLAM; k++) {
        WT[k * 6 + 0] = WT[k * 6 + 0] * rho;
        WT[k * 6 + 1] = WT[k * 6 + 1] / rho;
        WT[k * 6 + 2] = WT[k * 6 + 2] / rho;
        WT[k * 6 + 4] = WT[k * 6 + 4] / rho;
    }
    free(e);
}

int orc_vbt_weights_single(double x, double y, double hx, double hy, double rmin, double *WT, double *lms)
{
    vbt_tables *t = (vbt_tables *)malloc(sizeof(vbt_tables));
    vbt_init(rmin, t);
    vbt_weights_single_int(t, x, y, hx, hy, WT);
    if (lms) memcpy(lms, t->lms, sizeof(double) * NLAM);
    free(t);
    return 0;
}

/* rc_kernel_hankel_module.F90:31-38 weight indices and :47-54 G indices (0-based here) */
enum { RC_DXX = 0, RC_DXY = 1, RC_DYY = 2, RC_DX = 3, RC_DY = 4, RC_D0 = 5 };
enum { RG1 = 0, RG3DZ, RG2DZ, RG2DZ0, RG2G2DZZ, RG3, RG1DZ, RG2 };
/* const_module.F90:112-130 component slots; E: XX XY XZ YY YZ ZX ZY ZZ, H: XX XY XZ YX YZ ZX ZY */
enum { REXX = 0, REXY, REXZ, REYY, REYZ, REZX, REZY, REZZ };
enum { RHXX = 0, RHXY, RHXZ, RHYX, RHYZ, RHZX, RHZY };

typedef struct {
    double zrecv;
    int recv_layer, anom_cell;
} rc_recv_t;

/* rc_kernel_hankel_module.F90:181-225 Calc_Recv_Part; w1, w2 are [Nz+1][2] */
static void rc_recv_part(const bkg_t *b, const anom_t *an, double complex (*p)[2], double complex (*q)[2],
                         const double complex *eta, const rc_recv_t *rv, double complex (*w1)[2],
                         double complex (*w2)[2])
{
    int rl = rv->recv_layer, Nz = an->Nz;
    double complex eta_r = eta[rl];
    double complex eta_zr = eta_r * rv->zrecv;
    double complex eta_dr = rl > 1 ? eta_r * b->depth[rl - 1] * 2.0 : 0.0;
    int N = rv->anom_cell;
    int N1 = N + 1 > 1 ? N + 1 : 1;
    int N2 = N < Nz ? N : Nz;
    for (int i = N1; i <= Nz; i++) {
        int l = an->L[i];
        double complex e1 = cexp(-an->z[i - 1] * eta[l] + eta_zr);
        double complex e2 = cexp(-an->z[i - 1] * eta[l] - eta_zr + eta_dr);
        w1[i][0] = (e2 * p[rl][0] + e1);
        w1[i][1] = (-e2 * p[rl][0] + e1) * eta_r;
        w2[i][0] = (e2 * p[rl][1] + e1);
        w2[i][1] = (-e2 * p[rl][1] + e1) * eta_r;
    }
    if (rl < b->Nl) eta_dr = eta_r * b->depth[rl] * 2.0;
    else eta_dr = 1.0 * 1.7976931348623157e308; /* HUGE(zrecv) */
    for (int i = 1; i <= N2; i++) {
        int l = an->L[i];
        double complex e1 = cexp(an->z[i] * eta[l] - eta_zr);
        double complex e2 = cexp(an->z[i] * eta[l] + eta_zr - eta_dr);
        w1[i][0] = (e2 * q[rl][0] + e1);
        w1[i][1] = (e2 * q[rl][0] - e1) * eta_r;
        w2[i][0] = (e2 * q[rl][1] + e1);
        w2[i][1] = (e2 * q[rl][1] - e1) * eta_r;
    }
}

/* rc_kernel_hankel_module.F90:227-252 Calc_Ftb; Ftb is [Nz+1][3] */
static void rc_ftb(const anom_t *an, const double complex *expz, const double complex *eta,
                   double complex (*pq)[2], int N1, int N2, double complex (*Ftb)[3], double s)
{
    for (int i = N1; i <= N2; i++) {
        int l = an->L[i];
        double complex a = (1.0 - expz[i]);
        double complex a1 = a / eta[l];
        double complex e1[2], e2[2];
        for (int k = 0; k < 2; k++) {
            e1[k] = 1.0 + pq[i][k] * expz[i];
            e2[k] = (1.0 - pq[i][k] * expz[i]) * s;
        }
        Ftb[i][0] = a1 * e1[0];
        Ftb[i][1] = a1 * e1[1];
        Ftb[i][2] = a * e2[1];
    }
}

/* rc_kernel_hankel_module.F90:56-145 Calc_Integral_U with Calc_G_not_match (:147-179).
 * GE1 [Nz+1][8], GH1 [Nz+1][7] accumulate over lambda. */
static void rc_integral_u(const bkg_t *b, const anom_t *an, const rc_recv_t *rv, double lms, const double *W,
                          double complex (*GE1)[8], double complex (*GH1)[7])
{
    int Nl = b->Nl, Nz = an->Nz;
    double complex A[(Nl + 1) * (Nl + 1) * 2];
    double complex p[Nl + 1][2], q[Nl + 1][2], eta[Nl + 1], Arr[Nl + 1][2];
    double complex expz[Nz + 1], pez[Nz + 1][2], qez[Nz + 1][2], w1[Nz + 1][2], w2[Nz + 1][2], Ftb[Nz + 1][3];
    double lm2 = lms * lms;
    calc_apq(b, lms, Arr, p, q, eta, A);
    for (int iz = 1; iz <= Nz; iz++) expz[iz] = cexp(-eta[an->L[iz]] * (an->z[iz] - an->z[iz - 1]));
    rc_recv_part(b, an, p, q, eta, rv, w1, w2);
    memset(Ftb, 0, sizeof(Ftb));
    if (rv->anom_cell < 1) {
        calc_qexpz(b, an, expz, eta, q, qez);
        rc_ftb(an, expz, eta, qez, 1, Nz, Ftb, 1.0);
    } else if (rv->anom_cell > Nz) {
        calc_pexpz(b, an, expz, eta, p, pez);
        rc_ftb(an, expz, eta, pez, 1, Nz, Ftb, -1.0);
    } else {
        int N = rv->anom_cell;
        calc_pexpz(b, an, expz, eta, p, pez);
        calc_qexpz(b, an, expz, eta, q, qez);
        rc_ftb(an, expz, eta, pez, 1, N, Ftb, -1.0);
        rc_ftb(an, expz, eta, qez, N + 1, Nz, Ftb, 1.0);
    }
    int rl = rv->recv_layer;
    double complex csr = b->csigma[rl];
#define AIX(i, j, k) A[(((size_t)(i) * (Nl + 1)) + (j)) * 2 + (k)]
    for (int i = 1; i <= Nz; i++) {
        int l = an->L[i];
        double complex a1 = AIX(rl, l, 0), a2 = AIX(rl, l, 1);
        double complex *f = Ftb[i];
        double complex G[8];
        G[RG1] = a1 * f[0] * w1[i][0];
        G[RG3DZ] = (a2 * f[2] * w2[i][1]) / csr;
        G[RG2DZ] = (a2 * f[1] * w2[i][1]) / csr;
        G[RG2DZ0] = (a2 * f[2] * w2[i][0]) / csr;
        G[RG2G2DZZ] = lm2 * (a2 * f[1] * w2[i][0]) / csr;
        G[RG3] = (a2 * f[2] * w2[i][0] - a1 * f[0] * w1[i][1]);
        G[RG1DZ] = a1 * f[0] * w1[i][1];
        G[RG2] = a2 * f[1] * w2[i][0];
        double complex G11 = G[RG1] * b->iwm;
        GE1[i][REXX] = GE1[i][REXX] + G11 * W[RC_D0] + (G[RG3DZ] + G11) * W[RC_DXX];
        GE1[i][REXY] = GE1[i][REXY] + (G[RG3DZ] + G11) * W[RC_DXY];
        GE1[i][REXZ] = GE1[i][REXZ] + G[RG2DZ] * W[RC_DX];
        GE1[i][REYY] = GE1[i][REYY] + G11 * W[RC_D0] + (G[RG3DZ] + G11) * W[RC_DYY];
        GE1[i][REYZ] = GE1[i][REYZ] + G[RG2DZ] * W[RC_DY];
        GE1[i][REZX] = GE1[i][REZX] + G[RG2DZ0] * W[RC_DX];
        GE1[i][REZY] = GE1[i][REZY] + G[RG2DZ0] * W[RC_DY];
        GE1[i][REZZ] = GE1[i][REZZ] + G[RG2G2DZZ] * W[RC_D0];
        GH1[i][RHXX] = GH1[i][RHXX] + G[RG3] * W[RC_DXY];
        GH1[i][RHXY] = GH1[i][RHXY] + G[RG3] * W[RC_DYY] - G[RG1DZ] * W[RC_D0];
        GH1[i][RHXZ] = GH1[i][RHXZ] + G[RG2] * W[RC_DY];
        GH1[i][RHYX] = GH1[i][RHYX] + G[RG1DZ] * W[RC_D0] - G[RG3] * W[RC_DXX];
        GH1[i][RHYZ] = GH1[i][RHYZ] - G[RG2] * W[RC_DX];
        GH1[i][RHZX] = GH1[i][RHZX] - G[RG1] * W[RC_DY];
        GH1[i][RHZY] = GH1[i][RHZY] + G[RG1] * W[RC_DX];
    }
#undef AIX
}

#define RC_COMPS 15 /* 8 E slots then 7 H slots */

/* calc_rc_tensor_module.F90:161-229 CalcRecalculationGreenTensor3dElement for one receiver:
 * out[c][z] (stride Nr*Nz between components) */
static void rc_element(const vbt_tables *t, const bkg_t *b, const anom_t *an, const rc_recv_t *rv, double xs,
                       double ys, int lx, int ly, double dx, double dy, double complex *out, size_t comp_stride)
{
    int Nz = an->Nz;
    double *WT0 = (double *)malloc(sizeof(double) * NLAM * 6);
    double *WT = (double *)malloc(sizeof(double) * NLAM * 6);
    double s = 1.0 / 4.0 / PI_D;
    double x = lx * dx - dx / 2.0 + xs;
    double y = ly * dy - dy / 2.0 + ys;
    vbt_weights_single_int(t, x, y, dx, dy, WT0);
    double W0 = 0.0;
    for (int k = 0; k < NLAM; k++) {
        WT[k * 6 + RC_D0] = WT0[k * 6 + 0];
        WT[k * 6 + RC_DXX] = WT0[k * 6 + 1];
        WT[k * 6 + RC_DXY] = WT0[k * 6 + 2];
        WT[k * 6 + RC_DX] = WT0[k * 6 + 3];
        WT[k * 6 + RC_DYY] = WT0[k * 6 + 4];
        WT[k * 6 + RC_DY] = WT0[k * 6 + 5];
        for (int c = 0; c < 6; c++) if (fabs(WT[k * 6 + c]) > W0) W0 = fabs(WT[k * 6 + c]);
    }
    double complex (*GE1)[8] = (double complex (*)[8])calloc((size_t)(Nz + 1) * 8, sizeof(double complex));
    double complex (*GH1)[7] = (double complex (*)[7])calloc((size_t)(Nz + 1) * 7, sizeof(double complex));
    for (int k = 0; k < NLAM; k++) {
        double mx = 0;
        for (int c = 0; c < 6; c++) {
            double wm = fabs(WT[k * 6 + c] / W0);
            if (wm > mx) mx = wm;
        }
        if (mx > WT_THRESHOLD) {
            double lm = t->lms[k], W[6];
            W[RC_DXX] = WT[k * 6 + RC_DXX] / lm;
            W[RC_DYY] = WT[k * 6 + RC_DYY] / lm;
            W[RC_DXY] = WT[k * 6 + RC_DXY] / lm;
            W[RC_DX] = WT[k * 6 + RC_DX] * lm;
            W[RC_DY] = WT[k * 6 + RC_DY] * lm;
            W[RC_D0] = WT[k * 6 + RC_D0] * lm;
            rc_integral_u(b, an, rv, lm, W, GE1, GH1);
        }
    }
    for (int iz = 1; iz <= Nz; iz++) {
        for (int c = 0; c < 8; c++) out[(size_t)c * comp_stride + iz - 1] = GE1[iz][c] * s;
        for (int c = 0; c < 7; c++) out[(size_t)(8 + c) * comp_stride + iz - 1] = GH1[iz][c] * s;
    }
    free(GE1);
    free(GH1);
    free(WT);
    free(WT0);
}

/* calc_rc_tensor_module.F90:38-159 CalcRecalculationGreenTensor over the whole 2Nx x 2Ny lag plane (all
 * ranks' slabs): index ix < Nx is lag ix, ix > Nx is lag ix - 2Nx, ix = Nx is zero (same in y).
 * G is [2Ny][2Nx][15][Nr][Nz]; the receivers are those of orc_prepare_receivers. */
int orc_rc_tensor(const orc_model *m, int Nr, const double *zrecv, const double *x_shift, const double *y_shift,
                  const int *recv_layer, const int *anom_cell, double complex *G, int nthreads)
{
    int Nx = m->Nx, Ny = m->Ny, Nz = m->Nz;
    double *depth = (double *)malloc(sizeof(double) * (m->Nl + 1));
    double complex *k2 = (double complex *)malloc(sizeof(double complex) * (m->Nl + 1));
    bkg_t b;
    make_bkg(m, &b, depth, k2);
    int *L = (int *)malloc(sizeof(int) * (Nz + 1));
    orc_layer_numbers(m, L);
    double *dz = (double *)malloc(sizeof(double) * (Nz + 1));
    for (int i = 1; i <= Nz; i++) dz[i] = m->z[i] - m->z[i - 1];
    anom_t an = {Nz, L, m->z, dz};
    vbt_tables *t = (vbt_tables *)malloc(sizeof(vbt_tables));
    double rmin = sqrt(m->dx * m->dx + m->dy * m->dy) / 2.0; /* calc_rc_tensor_module.F90:80 */
    vbt_init(rmin, t);
    size_t E = (size_t)RC_COMPS * Nr * Nz;
    memset(G, 0, sizeof(double complex) * E * 4 * Nx * Ny);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) collapse(3)
#endif
    for (int iy = 0; iy < 2 * Ny; iy++)
        for (int ix = 0; ix < 2 * Nx; ix++)
            for (int r = 0; r < Nr; r++) {
                if (iy == Ny || ix == Nx) continue;
                int ly = iy < Ny ? iy : iy - 2 * Ny;
                int lx = ix < Nx ? ix : ix - 2 * Nx;
                rc_recv_t rv = {zrecv[r], recv_layer[r], anom_cell[r]};
                double complex *out = G + ((size_t)iy * 2 * Nx + ix) * E + (size_t)r * Nz;
                rc_element(t, &b, &an, &rv, x_shift[r], y_shift[r], lx, ly, m->dx, m->dy, out, (size_t)Nr * Nz);
            }
    free(t);
    free(dz);
    free(L);
    free(k2);
    free(depth);
    return 0;
}

/* The same for selected lag-plane indices only: out[n][15][Nr][Nz] for (ix[n], iy[n]) */
int orc_rc_tensor_lags(const orc_model *m, int Nr, const double *zrecv, const double *x_shift, const double *y_shift,
                       const int *recv_layer, const int *anom_cell, int n, const int *ixs, const int *iys,
                       double complex *out, int nthreads)
{
    int Nx = m->Nx, Ny = m->Ny, Nz = m->Nz;
    double *depth = (double *)malloc(sizeof(double) * (m->Nl + 1));
    double complex *k2 = (double complex *)malloc(sizeof(double complex) * (m->Nl + 1));
    bkg_t b;
    make_bkg(m, &b, depth, k2);
    int *L = (int *)malloc(sizeof(int) * (Nz + 1));
    orc_layer_numbers(m, L);
    double *dz = (double *)malloc(sizeof(double) * (Nz + 1));
    for (int i = 1; i <= Nz; i++) dz[i] = m->z[i] - m->z[i - 1];
    anom_t an = {Nz, L, m->z, dz};
    vbt_tables *t = (vbt_tables *)malloc(sizeof(vbt_tables));
    vbt_init(sqrt(m->dx * m->dx + m->dy * m->dy) / 2.0, t);
    size_t E = (size_t)RC_COMPS * Nr * Nz;
    memset(out, 0, sizeof(double complex) * E * n);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
#endif
    for (int k = 0; k < n; k++)
        for (int r = 0; r < Nr; r++) {
            int ix = ixs[k], iy = iys[k];
            if (iy == Ny || ix == Nx) continue;
            int ly = iy < Ny ? iy : iy - 2 * Ny;
            int lx = ix < Nx ? ix : ix - 2 * Nx;
            rc_recv_t rv = {zrecv[r], recv_layer[r], anom_cell[r]};
            rc_element(t, &b, &an, &rv, x_shift[r], y_shift[r], lx, ly, m->dx, m->dy, out + (size_t)k * E + (size_t)r * Nz,
                       (size_t)Nr * Nz);
        }
    free(t);
    free(dz);
    free(L);
    free(k2);
    free(depth);
    return 0;
}

/* The E and H sums of APPLY_RC_E_OP / APPLY_RC_H_OP (Continuation_Function_Module.F90:382-481) at one
 * point: g = tensor elements [15][Nr][Nz], u = currents [3][Nz]; o[f*3+c][Nr] with f = 0 (E), 1 (H). */
static void rc_point(int Nr, int Nz, const double complex *g, const double complex *u, double complex *o)
{
#define GG(c, r, z) g[((size_t)(c) * Nr + (r)) * Nz + (z)]
    for (int r = 0; r < Nr; r++) {
        double complex acc[6] = {0, 0, 0, 0, 0, 0};
        for (int z = 0; z < Nz; z++) {
            double complex ux = u[z], uy = u[Nz + z], uz = u[2 * Nz + z];
            acc[0] += GG(REXX, r, z) * ux + GG(REXY, r, z) * uy + GG(REXZ, r, z) * uz;
            acc[1] += GG(REXY, r, z) * ux + GG(REYY, r, z) * uy + GG(REYZ, r, z) * uz;
            acc[2] += GG(REZX, r, z) * ux + GG(REZY, r, z) * uy + GG(REZZ, r, z) * uz;
            acc[3] += GG(8 + RHXX, r, z) * ux + GG(8 + RHXY, r, z) * uy + GG(8 + RHXZ, r, z) * uz;
            acc[4] += GG(8 + RHYX, r, z) * ux - GG(8 + RHXX, r, z) * uy + GG(8 + RHYZ, r, z) * uz;
            acc[5] += GG(8 + RHZX, r, z) * ux + GG(8 + RHZY, r, z) * uy;
        }
        for (int o6 = 0; o6 < 6; o6++) o[(size_t)o6 * Nr + r] = acc[o6];
    }
#undef GG
}

/* currents j_c = (csiga - csigb(z)) E_c (LoadEint, Continuation_Function_Module.F90:240-263) as [y][x][3][Nz] */
static double complex *rc_currents(int Nx, int Ny, int Nz, const double complex *csiga, const double complex *csigb,
                                   const double complex *E)
{
    size_t cells = (size_t)Nx * Ny * Nz;
    double complex *j = (double complex *)malloc(sizeof(double complex) * 3 * cells);
    for (int y = 0; y < Ny; y++)
        for (int x = 0; x < Nx; x++)
            for (int c = 0; c < 3; c++)
                for (int z = 0; z < Nz; z++) {
                    size_t cell = ((size_t)z * Ny + y) * Nx + x;
                    double complex dsig = csiga[cell] - csigb[z];
                    j[(((size_t)y * Nx + x) * 3 + c) * Nz + z] = dsig * E[(size_t)c * cells + cell];
                }
    return j;
}

/* ReCalculation as direct lag sums over the spatial tensor: Ea, Ha are [Ny][Nx][3][Nr] (the reference's
 * Ea(Nr,3,Nx,Ny)); E is the anomaly field [3][Nz][Ny][Nx]. */
int orc_rc_apply_direct(int Nx, int Ny, int Nz, int Nr, const double complex *G, const double complex *csiga,
                        const double complex *csigb, const double complex *E, double complex *Ea,
                        double complex *Ha, int nthreads)
{
    size_t Et = (size_t)RC_COMPS * Nr * Nz;
    double complex *j = rc_currents(Nx, Ny, Nz, csiga, csigb, E);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
#endif
    for (int y = 0; y < Ny; y++)
        for (int x = 0; x < Nx; x++) {
            double complex *o = (double complex *)malloc(sizeof(double complex) * 6 * Nr);
            double complex *acc = (double complex *)calloc((size_t)6 * Nr, sizeof(double complex));
            for (int ys = 0; ys < Ny; ys++)
                for (int xs = 0; xs < Nx; xs++) {
                    int iy = (y - ys + 2 * Ny) % (2 * Ny), ix = (x - xs + 2 * Nx) % (2 * Nx);
                    rc_point(Nr, Nz, G + ((size_t)iy * 2 * Nx + ix) * Et, j + ((size_t)ys * Nx + xs) * 3 * Nz, o);
                    for (int k = 0; k < 6 * Nr; k++) acc[k] += o[k];
                }
            for (int c = 0; c < 3; c++)
                for (int r = 0; r < Nr; r++) {
                    Ea[(((size_t)y * Nx + x) * 3 + c) * Nr + r] = acc[(size_t)c * Nr + r];
                    Ha[(((size_t)y * Nx + x) * 3 + c) * Nr + r] = acc[(size_t)(3 + c) * Nr + r];
                }
            free(acc);
            free(o);
        }
    free(j);
    return 0;
}

/* ReCalculation through the 2Nx x 2Ny FFT as the reference does it: CalcFFTofRCTensor (:330-366) on the
 * spatial tensor, forward FFT of the currents, the point sums, backward FFT, division by 4NxNy (:324-328),
 * crop to the physical grid. */
int orc_rc_apply_fft(int Nx, int Ny, int Nz, int Nr, const double complex *G, const double complex *csiga,
                     const double complex *csigb, const double complex *E, double complex *Ea, double complex *Ha,
                     int nthreads)
{
    int n1 = 2 * Nx, n2 = 2 * Ny;
    size_t npts = (size_t)n1 * n2, Et = (size_t)RC_COMPS * Nr * Nz;
    double complex *Gh = (double complex *)malloc(sizeof(double complex) * npts * Et);
    double complex *U = (double complex *)calloc(npts * 3 * Nz, sizeof(double complex));
    double complex *O = (double complex *)malloc(sizeof(double complex) * npts * 6 * Nr);
    double complex *j = rc_currents(Nx, Ny, Nz, csiga, csigb, E);
    for (int y = 0; y < Ny; y++)
        for (int x = 0; x < Nx; x++)
            memcpy(U + ((size_t)y * n1 + x) * 3 * Nz, j + ((size_t)y * Nx + x) * 3 * Nz, sizeof(double complex) * 3 * Nz);
    free(j);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    /* element-wise 2-D transforms: plane[iy][ix] of one element */
#define RC_FFT_ELEMS(buf, ne, sign)                                                                       \
    do {                                                                                                  \
        _Pragma("omp parallel") {                                                                         \
            double complex *plane = (double complex *)malloc(sizeof(double complex) * npts);              \
            double complex *work = (double complex *)malloc(sizeof(double complex) * (n1 > n2 ? n1 : n2)); \
            _Pragma("omp for schedule(dynamic, 4)") for (size_t e = 0; e < (size_t)(ne); e++) {           \
                for (size_t p = 0; p < npts; p++) plane[p] = (buf)[p * (ne) + e];                         \
                fft2d(plane, n1, n2, (sign), work);                                                       \
                for (size_t p = 0; p < npts; p++) (buf)[p * (ne) + e] = plane[p];                         \
            }                                                                                             \
            free(work);                                                                                   \
            free(plane);                                                                                  \
        }                                                                                                 \
    } while (0)
    memcpy(Gh, G, sizeof(double complex) * npts * Et);
    RC_FFT_ELEMS(Gh, Et, -1);
    RC_FFT_ELEMS(U, (size_t)3 * Nz, -1);
    for (size_t p = 0; p < npts; p++) rc_point(Nr, Nz, Gh + p * Et, U + p * 3 * Nz, O + p * 6 * Nr);
    RC_FFT_ELEMS(O, (size_t)6 * Nr, 1);
#undef RC_FFT_ELEMS
    double complex nrm = (double)(4 * Nx * Ny);
    for (int y = 0; y < Ny; y++)
        for (int x = 0; x < Nx; x++)
            for (int c = 0; c < 3; c++)
                for (int r = 0; r < Nr; r++) {
                    const double complex *o = O + ((size_t)y * n1 + x) * 6 * Nr;
                    Ea[(((size_t)y * Nx + x) * 3 + c) * Nr + r] = o[(size_t)c * Nr + r] / nrm;
                    Ha[(((size_t)y * Nx + x) * 3 + c) * Nr + r] = o[(size_t)(3 + c) * Nr + r] / nrm;
                }
    free(O);
    free(U);
    free(Gh);
    return 0;
}

/* sources_module.F90:26-66 PlaneWave: normal field at receiver depths, F[Nr][6] = Ex Ey Ez Hx Hy Hz;
 * pol 0 = EX, 1 = EY */
int orc_plane_wave_points(const orc_model *m, int pol, int Nr, const double *zrecv, double complex *F)
{
    int Nl = m->Nl;
    double depth[Nl + 1];
    double complex k2[Nl + 1];
    bkg_t b;
    make_bkg(m, &b, depth, k2);
    double complex Arr[Nl + 1][2], p[Nl + 1][2], q[Nl + 1][2], eta[Nl + 1];
    double complex *A = (double complex *)calloc((size_t)(Nl + 1) * (Nl + 1) * 2, sizeof(double complex));
    calc_apq(&b, 0.0, Arr, p, q, eta, A);
#define AIX(i, j, k) A[(((size_t)(i) * (Nl + 1)) + (j)) * 2 + (k)]
    double complex t1 = Nl > 1 ? 1.0 + q[1][0] * cexp(-b.depth[1] * eta[1] * 2.0) : 1.0;
    t1 = AIX(1, 1, 0) * t1;
    memset(F, 0, sizeof(double complex) * 6 * Nr);
    for (int ir = 0; ir < Nr; ir++) {
        int l = orc_get_layer(zrecv[ir], Nl, depth);
        if (l < 1) l = 1;
        double complex t2 = AIX(l, 1, 0) / t1;
        double complex e1 = cexp(-eta[l] * zrecv[ir]);
        double complex e2 = l < Nl ? q[l][0] * (cexp(-eta[l] * (2.0 * b.depth[l] - zrecv[ir]))) : 0.0;
        double complex g1 = t2 * (e1 + e2);
        double complex g2 = -t2 * (e1 - e2) * eta[l] / b.iwm;
        if (pol == 0) {
            F[ir * 6 + 0] = g1;
            F[ir * 6 + 4] = g2;
        } else {
            F[ir * 6 + 1] = g1;
            F[ir * 6 + 3] = -g2;
        }
    }
#undef AIX
    free(A);
    return 0;
}
