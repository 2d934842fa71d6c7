// Receiver continuation (fields at receiver points from the anomaly's currents): internal interface
// between the C ABI (capi.cu) and the kernels (continuation.cu).
#pragma once
#include <cuda_runtime.h>

struct RcOp;

struct RcReceiver {
    double zrecv;     // depth after PrepareRecvs (moved to the top of its cell when strictly inside one)
    double x_shift, y_shift;
    int recv_layer;   // >= 1
    int anom_cell;    // anomaly cells above the receiver: 0 above the anomaly, Nz+1 below it
};

// z: Nz+1 cell borders; receivers already prepared (PrepareRecvs)
RcOp *rc_create(int Nx, int Ny, int Nz, double dx, double dy, const double *z, int Nr, const RcReceiver *recv);
// CalcRecalculationGreenTensor: csigma [Nl+1] (air first), thick [Nl-1], Lnumber [Nz+1]
int rc_calc_kernel(RcOp *op, int Nl, const double2 *csigma, const double *thick, double omega, const int *Lnumber);
// CalcFFTofRCTensor: the spatial tensor becomes its 2Nx x 2Ny spectrum in place
int rc_fft_kernel(RcOp *op);
// FinalizeRCOperator: csiga complex [Nz][Ny][Nx] (x fastest), host memory
int rc_set_anomaly_conductivity(RcOp *op, const double2 *csiga_host);
// ReCalculation on device buffers: E [3][Nz][Ny][Nx] -> Ea, Ha [Ny][Nx][3][Nr]
int rc_recalculate_device(RcOp *op, const double2 *dE, double2 *dEa, double2 *dHa);
// the same with host buffers (staged through the operator's device buffers)
int rc_recalculate_host(RcOp *op, const double2 *E, double2 *Ea, double2 *Ha);
// current tensor (spatial before rc_fft_kernel, spectral after) to host: [2Ny][2Nx][15][Nr][Nz]
int rc_copy_kernel(RcOp *op, double2 *host);
int rc_receivers(const RcOp *op, RcReceiver *out);
int rc_count(const RcOp *op);
int rc_nz(const RcOp *op);
const double *rc_borders(const RcOp *op);
cudaStream_t rc_stream(const RcOp *op);
void rc_delete(RcOp *op);
