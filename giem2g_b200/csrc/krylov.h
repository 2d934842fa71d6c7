// GPU nested FGMRES (GFGMRES/gmres.F90, seq_fgmres.F90) on one IE operator.
#pragma once
#include "ie_internal.h"

void krylov_free(IeOp *op);
// SolveEquation on device vectors (complex128, (Nx,Ny,Nz,3)); d_E0 may be null
int krylov_solve_device(IeOp *op, const double2 *d_Ebkg, double2 *d_Esol, const double2 *d_E0,
                        const GIEM2G_FGMRES_CTL &ctl, GIEM2G_RESULT *info);
int krylov_history(IeOp *op, double *out, int max_len);
