// Internal state of one IE operator on one GPU, and the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "../../include/giem2g.h"

enum { G2_OK = 0, G2_ERR_ARG = -1, G2_ERR_CUDA = -2, G2_ERR_STATE = -3, G2_ERR_UNSUPPORTED = -4,
       G2_ERR_NUMERIC = -5, G2_ERR_NOMEM = -6 };

struct ApplyScratch {
    void *U1 = nullptr;    // [2Nx][3Nz][Ny]   x-spectrum / inverse-y output
    void *Uhat = nullptr;  // [Nx][Ny][4][3Nz] full 2-D spectrum in (kx-pair, ky-pair, slot) order
};

struct IeOp {
    // geometry
    int Nx = 0, Ny = 0, Nz = 0;
    double dx = 0, dy = 0;
    std::vector<double> z, dz;
    // background (complex conductivity per layer, index 0 = air)
    int Nl = 0;
    std::vector<double2> csigma;
    std::vector<double> thick;
    double omega = 0;
    std::vector<int> Lnumber;          // 0..Nz
    std::vector<double2> csigb;        // per cell layer
    std::vector<double> sqsigb;
    bool have_background = false;
    bool have_spatial = false, have_spectral = false, have_sigma = false;
    // device data
    double2 *d_spatial = nullptr;      // [Nx][Ny][Tunit] FP64 spatial tensor
    double2 *d_tensor64 = nullptr;     // [Nx][Ny][Tunit] FP64 spectral tensor
    float2 *d_tensor32 = nullptr;      // same, complex64 copy
    double2 *d_csiga = nullptr;        // [Nz][Ny][Nx]
    double2 *d_gsig64 = nullptr, *d_asig64 = nullptr;  // per-cell pre/post coefficients
    float2 *d_gsig32 = nullptr, *d_asig32 = nullptr;
    double *d_post64 = nullptr;        // [2][Nz]: sqrt(Re sigma_b), 1/(dz*4NxNy)
    float *d_post32 = nullptr;
    double2 *d_twx64 = nullptr, *d_twy64 = nullptr;
    float2 *d_twx32 = nullptr, *d_twy32 = nullptr;
    ApplyScratch scratch;
    ApplyScratch pair_scratch;         // two complex64 vectors per apply (allocated on first paired apply)
    int *d_err = nullptr;              // device error word written by bounded waits (0 = ok)
    void *krylov = nullptr;            // solver workspace (krylov.cu)
    // host staging for the reference-facing (host-pointer) apply
    double2 *h_stage_in = nullptr, *h_stage_out = nullptr;
    double2 *d_vin = nullptr, *d_vout = nullptr;
    float2 *d_vin32 = nullptr, *d_vout32 = nullptr;  // complex64 copies for the mode-1 host apply
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // events around the contraction launch of eager device applies (giem2g_set_kernel_timing)
    bool time_contract = false;
    cudaEvent_t evc0 = nullptr, evc1 = nullptr;
    int precision_mode = 0;            // 0 plain FP64, 1 mixed (c64 inner)
    bool use_fast_contract = true;     // GIEM2G_GENERIC_CONTRACT=1 selects the generic contraction kernel
    int contract_variant[3] = {0, 0, 0};  // tile-shape variant: FP64, complex64, paired complex64
    // fused y-transforms + contraction (ypipe.cu) per form: its variant, or -1 for the separate passes
    // (k_fy, contraction, k_by).  The separate passes are the default (faster at 128x128x32 on a B200);
    // the fused pass is a tile-shape variant the autotuner may pick where ie_ypipe_supported holds.
    int ypipe_mode[3] = {-1, -1, -1};
    int fft_lines[2] = {32, 32};          // lines per CTA of the FFT passes, complex128 / complex64 (autotuned)
    long long config_gen = 0;             // bumped on every launch-shape change; captured graphs compare it
    // outer right-preconditioner hook (learned preconditioner): 0 off, 1 warm-starts the inner GMRES,
    // 2 replaces it
    int precond_mode = 0;
    int (*precond_fn)(void *, const void *, void *, long long, void *) = nullptr;
    void *precond_user = nullptr;
    void *learned = nullptr;           // network of giem2g_set_preconditioner (learned_net.cu), owned
    // counters (Integral_Equation_Module.F90:44-56)
    long long mult_num = 0;
    double apply_seconds = 0;
    int last_kernel_launches = 0;

    int P() const { return Nz * (Nz + 1) / 2; }
    int Tunit() const { return 4 * P() + 2 * Nz * Nz; }
    size_t units() const { return (size_t)Nx * Ny; }
    size_t cells() const { return (size_t)Nx * Ny * Nz; }
    size_t nvec() const { return 3 * cells(); }
};

// apply.cu
// gate: optional device flag; when it reads 0 every kernel of the apply returns at once (used by the
// solver to skip Arnoldi steps after convergence without a host round trip)
int ie_apply_device64(IeOp *op, const double2 *d_in, double2 *d_out, cudaStream_t st, const int *gate = nullptr);
int ie_apply_device32(IeOp *op, const float2 *d_in, float2 *d_out, cudaStream_t st, const int *gate = nullptr);
// complex128 in/out, complex64 apply inside (giem2g_set_precision mode 1)
int ie_apply_host_mixed(IeOp *op, const double2 *d_in, double2 *d_out, cudaStream_t st);
// The same apply over caller-given scratch (U1: first n_u1 elements, Uhat: the rest).
size_t ie_apply_scratch_elems(const IeOp *op, size_t *n_u1);
int ie_apply_device64_scratch(IeOp *op, const double2 *d_in, double2 *d_out, cudaStream_t st, double2 *U1,
                              double2 *Uhat);
int ie_apply_device32_scratch(IeOp *op, const float2 *d_in, float2 *d_out, cudaStream_t st, float2 *U1,
                              float2 *Uhat);
// Two complex64 vectors of one operator per apply (shared tensor reads); scratch holds twice the
// single-vector intermediates.  G2_ERR_UNSUPPORTED when the grid has no paired contraction.
size_t ie_pair_scratch_elems(const IeOp *op, size_t *n_u1);
int ie_pair_scratch(IeOp *op, float2 **U1, float2 **Uh);
int ie_apply_pair32(IeOp *op, const float2 *in0, const float2 *in1, float2 *out0, float2 *out1, cudaStream_t st,
                    float2 *U1, float2 *Uh);
bool ie_contract_pair32_supported(int Nx, int Ny, int Nz);
int ie_contract_pair32(const float2 *G, float2 *Uhat, int Nx, int Ny, int Nz, int *err, cudaStream_t st,
                       const int *gate, int variant);
int ie_contract_pair_variants(int Nz);
// Process-wide static scratch of the static-scratch apply: device address (set-up on first use per
// device) and capacity in bytes.
int ie_static_scratch(void **ptr, size_t *capacity);
// 3x3x3 convolution data movement (channels-last): im2col (bf16) and its gather-form adjoint (fp32)
int ie_im2col3d(const void *x, void *cols, int N, int D, int H, int W, int C, int s, int Kp, cudaStream_t st);
int ie_col2im3d(const float *dcols, float *dx, int N, int D, int H, int W, int C, int s, int Kp, cudaStream_t st);
// BF16 tensor-core GEMM, FP32 out: C = A B^T (or C += A B^T), A [M][K], B [N][K] K-major
int ie_gemm_bf16_tn(const void *A, const void *B, float *C, int M, int N, int K, int lda, int ldb, int ldc,
                    int accumulate, int *err, cudaStream_t st);
int ie_alloc_scratch(IeOp *op);
int ie_make_twiddles(IeOp *op);
// kernels one apply launches in a form (0 FP64, 1 complex64, 2 paired complex64)
int ie_kernel_launch_count_apply(const IeOp *op, int form);

// ypipe.cu: forward y-FFT, contraction and inverse y-FFT in one persistent kernel (U1 in, U1 out, the
// spectrum Uh as scratch, `state` = ie_ypipe_state_bytes of counters zeroed by the launcher)
bool ie_ypipe_supported(int Nx, int Ny, int Nz);
int ie_ypipe_variants(int form);
size_t ie_ypipe_state_bytes(int Nx);
int ie_ypipe(IeOp *op, int form, const void *G, void *U1, void *Uh, int *state, cudaStream_t st, const int *gate);

// learned_net.cu: the U-Net outer preconditioner (kind 0 off, 1 warm start, 2 replace)
int ie_set_learned_preconditioner(IeOp *op, int kind, const char *weights_path);
long long ie_learned_calls(const IeOp *op);
int ie_learned_apply(IeOp *op, const double2 *d_v, double2 *d_z);
void ie_free_learned(IeOp *op);

// green.cu: spatial Green's tensor (FP64) into op->d_spatial
int ie_green_tensor(IeOp *op, cudaStream_t st);

// contract.cu: specialised contraction; G2_ERR_UNSUPPORTED when Nz has no specialisation
int ie_contract_fast64(const double2 *G, double2 *Uhat, int Nx, int Ny, int Nz, int *err, cudaStream_t st, int variant,
                       const int *gate);
int ie_contract_fast32(const float2 *G, float2 *Uhat, int Nx, int Ny, int Nz, int *err, cudaStream_t st, int variant,
                       const int *gate);
int ie_contract_variants(int precision, int Nz);

// tensor_fft.cu
int ie_tensor_spectrum(IeOp *op, cudaStream_t st);

// sigma.cu (in apply.cu)
int ie_prepare_sigma(IeOp *op, cudaStream_t st);

int ie_check_device_error(IeOp *op);  // reads d_err after a sync; nonzero -> G2_ERR_NUMERIC
void g2_count_launches(int n);          // cumulative count of this library's kernel launches
long long g2_launch_total();
void g2_log(const char *msg);
void g2_set_error(const char *file, int line, const char *msg);
void g2_set_error_msg(const std::string &msg);
