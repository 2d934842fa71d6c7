/* A plain C host of the library (no Python): the call sequence of the reference's C interface
 * (giem2g_interfaces.F90) plus giem2g_solve, then the receiver fields, on a 16x16x8 block model.
 * Prints one line "iterations stat true_residual recomputed_residual receiver_max" and exits 0 when the
 * solution satisfies the system to the solver's tolerance. */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "giem2g.h"

#define NX 16
#define NY 16
#define NZ 8

static double nrm(const double complex *v, size_t n)
{
    double s = 0;
    for (size_t i = 0; i < n; i++) s += creal(v[i] * conj(v[i]));
    return sqrt(s);
}

int main(void)
{
    const double pi = 3.14159265358979323846, mu0 = 4e-7 * pi, eps0 = 1.0 / (mu0 * 299792458.0 * 299792458.0);
    const double freq = 1.0, omega = 2 * pi * freq;
    double z[NZ + 1], dz[NZ];
    for (int i = 0; i <= NZ; i++) z[i] = 50.0 * i;
    for (int i = 0; i < NZ; i++) dz[i] = z[i + 1] - z[i];
    GIEM2G_ANOMALY_TYPE an = {NX, NY, NZ, 100.0, 100.0, z, dz};
    GIEM2G_DATA_TYPE d;
    giem2g_calc_data_sizes(an, &d);
    giem2g_prepare_ie_kernel(an, d);
    if (giem2g_last_status()) { fprintf(stderr, "prepare: %s\n", giem2g_last_error()); return 1; }
    void *ie = d.giem2g_tensor;
    const double sig_l[3] = {0.01, 0.001, 0.1}, thick[2] = {500.0, 1500.0};
    double complex csigb_l[4];
    csigb_l[0] = 1e-12 - I * omega * eps0;
    for (int l = 0; l < 3; l++) csigb_l[l + 1] = sig_l[l] - I * omega * eps0;
    GIEM2G_BACKGROUND_TYPE bkg = {3, csigb_l, (void *)thick};
    giem2g_calc_ie_kernel(ie, bkg, an, omega);
    giem2g_calc_fft_of_ie_kernel(ie);
    if (giem2g_last_status()) { fprintf(stderr, "kernel: %s\n", giem2g_last_error()); return 1; }
    const size_t cells = (size_t)NX * NY * NZ, n = 3 * cells;
    double complex *csiga = malloc(sizeof(double complex) * cells);
    for (int k = 0; k < NZ; k++)
        for (int j = 0; j < NY; j++)
            for (int i = 0; i < NX; i++) {
                const int blk = i >= 5 && i < 11 && j >= 4 && j < 12 && k >= 2 && k < 6;
                csiga[((size_t)k * NY + j) * NX + i] = (blk ? 0.5 : 0.01) - I * omega * eps0;
            }
    giem2g_set_anomaly_conductivity(ie, csiga);
    double complex *E0 = calloc(n, sizeof(double complex)), *E = malloc(sizeof(double complex) * n);
    for (size_t c = 0; c < cells; c++) E0[c] = 1.0; /* uniform Ex */
    GIEM2G_FGMRES_CTL ctl = {1e-8, 100, 10, 30, 0};
    GIEM2G_RESULT res;
    if (giem2g_solve(ie, E0, E, NULL, ctl, &res)) { fprintf(stderr, "solve: %s\n", giem2g_last_error()); return 1; }
    /* the system: chi = E / a, A chi = sqrt(Re sigma_b) E0 with a = 2 sqrt(Re sigma_b) / (sigma_a + conj sigma_b) */
    double complex *chi = malloc(sizeof(double complex) * n), *Ax = malloc(sizeof(double complex) * n);
    double complex *rhs = malloc(sizeof(double complex) * n);
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < NZ; k++) {
            const double complex sb = csigb_l[1]; /* every cell lies in the first layer (z < 500 m) */
            const double s = sqrt(creal(sb));
            for (size_t p = 0; p < (size_t)NX * NY; p++) {
                const size_t cell = (size_t)k * NX * NY + p, i = (size_t)c * cells + cell;
                const double complex a = 2.0 * s / (csiga[cell] + conj(sb));
                chi[i] = E[i] / a;
                rhs[i] = s * E0[i];
            }
        }
    giem2g_apply_ie_operator(ie, chi, Ax);
    for (size_t i = 0; i < n; i++) Ax[i] -= rhs[i];
    const double rres = nrm(Ax, n) / nrm(rhs, n);
    /* receiver fields at the surface from this solution */
    const double zr = 0.0, xs = 0.0, ys = 0.0;
    void *rc = giem2g_rc_create(bkg, an, 1, &zr, &xs, &ys);
    double rmax = -1;
    if (rc && !giem2g_rc_calc_kernel(rc, bkg, omega) && !giem2g_rc_calc_fft_of_kernel(rc) &&
        !giem2g_rc_set_anomaly_conductivity(rc, csiga)) {
        double complex *Ea = malloc(sizeof(double complex) * NX * NY * 3), *Ha = malloc(sizeof(double complex) * NX * NY * 3);
        if (!giem2g_rc_recalculate(rc, E, Ea, Ha)) {
            rmax = 0;
            for (int i = 0; i < NX * NY * 3; i++) {
                if (!isfinite(creal(Ea[i])) || !isfinite(cimag(Ha[i]))) rmax = NAN;
                if (cabs(Ea[i]) > rmax) rmax = cabs(Ea[i]);
            }
        }
        free(Ea);
        free(Ha);
    }
    giem2g_rc_delete(rc);
    printf("%d %d %.3e %.3e %.6e\n", res.iterations, res.stat, res.be, rres, rmax);
    giem2g_delete_ie_operator(ie);
    free(csiga); free(E0); free(E); free(chi); free(Ax); free(rhs);
    return (res.stat == 1 && rres < 1.5e-8 && rmax > 0) ? 0 : 2;
}
