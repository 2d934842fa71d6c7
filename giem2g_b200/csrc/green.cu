// Green's tensor construction on the GPU -- placeholder.
#include "common.cuh"
#include "ie_internal.h"

int ie_green_tensor(IeOp *op, cudaStream_t st)
{
    (void)op; (void)st;
    g2_set_error_msg("Green's tensor construction on the GPU is not built yet");
    return G2_ERR_UNSUPPORTED;
}
