// GPU nested FGMRES -- placeholder until the device solver lands.
#include "common.cuh"
#include "krylov.h"

void krylov_free(IeOp *op) { (void)op; }

extern "C" int giem2g_solve(void *, const void *, void *, const void *, GIEM2G_FGMRES_CTL, GIEM2G_RESULT *)
{
    return G2_ERR_UNSUPPORTED;
}
extern "C" int giem2g_solve_device(void *, const void *, void *, const void *, GIEM2G_FGMRES_CTL, GIEM2G_RESULT *)
{
    return G2_ERR_UNSUPPORTED;
}
extern "C" int giem2g_get_misfit_history(void *, double *, int) { return 0; }
