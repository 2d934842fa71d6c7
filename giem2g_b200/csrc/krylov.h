// GPU nested FGMRES (GFGMRES/gmres.F90, seq_fgmres.F90) on one IE operator.
#pragma once
#include "ie_internal.h"

void krylov_free(IeOp *op);
