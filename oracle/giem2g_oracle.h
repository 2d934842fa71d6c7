/*
 * giem2g_oracle.h -- CPU FP64 restatement of GIEM2G's integral-equation solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the correctness oracle for the
 * B200 kernels.  Only the test-suite, the smoke check and the CPU-baseline leg of
 * the benchmark load it; the product library never links or calls it.
 *
 * Every entry point restates a reference routine (file:line given at each
 * definition in giem2g_oracle.c).  Complex numbers are C99 `double complex`
 * (same memory layout as Fortran COMPLEX(8) and numpy complex128).
 *
 * Array layouts (all C row-major statements of the reference's Fortran layouts):
 *   field vectors  v[c][z][y][x]      == Fortran v(Nx,Ny,Nz,3)      (x fastest)
 *   conductivity   csiga[z][y][x]     == Fortran csiga(Nx,Ny,Nz)
 *   spatial tensor symm[lx][ly][4][P] == Fortran G_symm(P,4,Ny,Nx),  P = Nz(Nz+1)/2,
 *                                        packed upper: (i,j), i<=j -> i + j(j+1)/2
 *                  asym[lx][ly][2][Nz*Nz] == Fortran G_asym(Nz,Nz,2,Ny,Nx), column-major
 *                  component order symm: xx, xy, yy, zz   asym: xz, yz
 *   spectral tensor, same shapes indexed [kx-pair q][ky r] for q<Nx, r<Ny.
 *
 * Parity status: the reference ships no tests, golden vectors or fixtures and
 * cannot be built here (Fortran + MPI + FFTW).  Parity is therefore UNPINNED
 * against reference outputs; it is anchored on a dense block-Toeplitz brute
 * force (orc_apply_toeplitz) and on an independent numpy restatement.
 */
#ifndef GIEM2G_ORACLE_H
#define GIEM2G_ORACLE_H
#include <complex.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int Nx, Ny, Nz;
    double dx, dy;
    const double *z;       /* Nz+1 cell borders (depth, m, positive down) */
    int Nl;                /* number of background layers (half-space included) */
    const double complex *csigma; /* Nl+1, index 0 = air (complex conductivity) */
    const double *thick;   /* Nl-1 layer thicknesses */
    double omega;          /* angular frequency */
} orc_model;

typedef struct {
    int iterations;
    double bea;            /* Arnoldi misfit */
    double be;             /* true misfit */
    int stat;              /* 1 CONVERGED, 2 NON_TRUE_CONVERGED, -1 NON_CONVERGED */
    int applies;           /* operator applications performed */
} orc_result;

/* Layer helpers (data_types_module.F90) */
int orc_get_layer(double z, int Nl, const double *depth);
void orc_layer_numbers(const orc_model *m, int *Lnumber /* Nz+1 */);
void orc_background_cells(const orc_model *m, double complex *csigb /*Nz*/, double *sqsigb /*Nz*/);

/* VolumeBesselTransforms.F90 weights for one lag (exposed for testing) */
int orc_vbt_weights(double x, double y, double hx, double hy, double rmin,
                    double *WT /* [501][6] */, double *lms /* [501] */);

/* Spatial Green's tensor (calc_ie_tensor_module.F90:54) */
int orc_green_tensor(const orc_model *m, double complex *symm, double complex *asym, int nthreads);

/* Spectral transform of the tensor (Integral_Equation_Module.F90:319) */
int orc_tensor_spectrum(int Nx, int Ny, int Nz,
                        const double complex *symm, const double complex *asym,
                        double complex *symm_hat, double complex *asym_hat, int nthreads);

/* Operator apply (apply_ie_operator_module.F90:39) from the spectral tensor */
int orc_apply(int Nx, int Ny, int Nz,
              const double complex *symm_hat, const double complex *asym_hat,
              const double complex *csiga, const double complex *csigb,
              const double *sqsigb, const double *dz,
              const double complex *v_in, double complex *v_out, int nthreads);

/* Dense block-Toeplitz brute force of the same operator from the SPATIAL tensor */
int orc_apply_toeplitz(int Nx, int Ny, int Nz,
                       const double complex *symm, const double complex *asym,
                       const double complex *csiga, const double complex *csigb,
                       const double *sqsigb, const double *dz,
                       const double complex *v_in, double complex *v_out);

/* Plane-wave right-hand side (sources_module.F90:67); pol 0 = EX, 1 = EY */
int orc_plane_wave(const orc_model *m, int pol, double complex *E0 /* [3][Nz][Ny][Nx] */);

/* SolveEquation (ie_solver_module.F90:43) with nested FGMRES (GFGMRES/gmres.F90) */
int orc_solve(int Nx, int Ny, int Nz,
              const double complex *symm_hat, const double complex *asym_hat,
              const double complex *csiga, const double complex *csigb,
              const double *sqsigb, const double *dz,
              const double complex *E_bkg, const double complex *E0_guess /* may be NULL */,
              int outer_buf, int inner_buf, int max_restart, double tol,
              double complex *Esol, orc_result *info,
              double *misfit_history /* may be NULL; outer Arnoldi misfits */, int history_len,
              int nthreads);

/* csiga from a real conductivity in file order siga[y][x][z] (ie_solver_module.F90:116) */
void orc_set_anomaly_sigma(int Nx, int Ny, int Nz, const double *siga_zxy, double freq,
                           int displacement_currents, double complex *csiga);

/* complex conductivity of the background for a frequency (data_types_module.F90:244) */
void orc_set_freq(int Nl, const double *sigma, double freq, int displacement_currents,
                  double complex *csigma /* Nl+1 */);

/* Receiver continuation (Continuation_Function_Module.F90, calc_rc_tensor_module.F90,
 * rc_kernel_hankel_module.F90).  Receivers: depth zrecv (moved to the top of its cell when strictly inside
 * one), lateral shifts x_shift, y_shift, layer and anom_cell from orc_prepare_receivers.
 * Tensor layout [2Ny][2Nx][15][Nr][Nz]: lag index ix < Nx is lag ix, ix > Nx is ix - 2Nx, ix = Nx is zero
 * (same in y); components E: xx xy xz yy yz zx zy zz, then H: xx xy xz yx yz zx zy.
 * Fields at receivers: Ea, Ha [Ny][Nx][3][Nr] (the reference's Ea(Nr,3,Nx,Ny)). */
int orc_prepare_receivers(const orc_model *m, int Nr, double *zrecv, int *recv_layer, int *anom_cell);
int orc_vbt_weights_single(double x, double y, double hx, double hy, double rmin,
                           double *WT /* [501][6] */, double *lms /* [501] */);
int orc_rc_tensor(const orc_model *m, int Nr, const double *zrecv, const double *x_shift, const double *y_shift,
                  const int *recv_layer, const int *anom_cell, double complex *G, int nthreads);
int orc_rc_tensor_lags(const orc_model *m, int Nr, const double *zrecv, const double *x_shift, const double *y_shift,
                       const int *recv_layer, const int *anom_cell, int n, const int *ix, const int *iy,
                       double complex *out /* [n][15][Nr][Nz] */, int nthreads);
int orc_rc_apply_direct(int Nx, int Ny, int Nz, int Nr, const double complex *G, const double complex *csiga,
                        const double complex *csigb, const double complex *E, double complex *Ea,
                        double complex *Ha, int nthreads);
int orc_rc_apply_fft(int Nx, int Ny, int Nz, int Nr, const double complex *G, const double complex *csiga,
                     const double complex *csigb, const double complex *E, double complex *Ea, double complex *Ha,
                     int nthreads);
/* PlaneWave (sources_module.F90:26-66) at receiver depths: F[Nr][6] = Ex Ey Ez Hx Hy Hz; pol 0 EX, 1 EY */
int orc_plane_wave_points(const orc_model *m, int pol, int Nr, const double *zrecv, double complex *F);

double orc_eps0(void);
double orc_mu0(void);

#ifdef __cplusplus
}
#endif
#endif
