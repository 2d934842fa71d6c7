// GPU nested FGMRES (GFGMRES/gmres.F90, seq_fgmres.F90) on one IE operator.
#pragma once
#include "ie_internal.h"

void krylov_free(IeOp *op);
// SolveEquation on device vectors (complex128, (Nx,Ny,Nz,3)); d_E0 may be null
int krylov_solve_device(IeOp *op, const double2 *d_Ebkg, double2 *d_Esol, const double2 *d_E0,
                        const GIEM2G_FGMRES_CTL &ctl, GIEM2G_RESULT *info);
int krylov_history(IeOp *op, double *out, int max_len);

// Batched solves: n instances (operator, right-hand side) in lockstep on ops[0]'s stream.
int batch_create(IeOp *const *ops, int n, int mo, int mi, int precision, void **out);
void batch_free(void *b);
int batch_solve_device(void *b, const double2 *const *d_Ebkg, double2 *const *d_Esol, const double2 *const *d_E0,
                       const GIEM2G_FGMRES_CTL &ctl, GIEM2G_RESULT *info);
int batch_history(void *b, int i, double *out, int max_len);
// device staging for host-array solves: 3n vectors of N complex128 (E_bkg[i] at i*N, E_sol[i] at (n+i)*N,
// E0[i] at (2n+i)*N)
int batch_stage(void *b, double2 **d_stage, size_t *N);
int batch_size(void *b);
IeOp *batch_op(void *b, int i);
