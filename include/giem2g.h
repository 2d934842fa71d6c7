/*
 * giem2g.h -- C ABI of the B200 implementation of GIEM2G's integral-equation solve path.
 *
 * The first block re-exports the nine BIND(C) entry points of the reference's
 * C interface with identical names, argument lists and struct layouts, so a host
 * that links the reference's libgiem2g can link this library instead.  Citations
 * are to giem2g_interfaces.F90 in the GIEM2G source tree.
 *
 * Differences from the reference that a caller can observe:
 *   - One process drives one GPU; the communicator in GIEM2G_DATA_TYPE.comm64 is
 *     ignored and every array covers the whole anomaly (Ny_loc == Ny).
 *   - The caller-allocated kernel/FFT buffers named in GIEM2G_DATA_TYPE are not
 *     used (their sizes are still reported); the tensor and spectra live on the GPU.
 *   - giem2g_set_anomaly_conductivity copies csiga to the GPU at call time (the
 *     reference keeps a pointer to the caller's array and re-reads it on every
 *     apply); call it again after changing csiga.
 *   - Errors are recorded: giem2g_last_status() returns 0 or a negative code and
 *     giem2g_last_error() the message.  The reference has no error return.
 *   - Nx and Ny must be even with 2*Nx and 2*Ny powers of two (4..1024).
 *
 * Vectors are complex(8) (Nx,Ny,Nz,3), x fastest, components (Ex,Ey,Ez).
 */
#ifndef GIEM2G_H
#define GIEM2G_H

#ifdef __cplusplus
extern "C" {
#endif

/* giem2g_interfaces.F90:33-37 */
typedef struct {
    int Nl;              /* number of layers (half-space included) */
    void *csigb;         /* Nl+1 complex(8): [0] = air, then layers */
    void *thickness;     /* Nl-1 real(8) */
} GIEM2G_BACKGROUND_TYPE;

/* giem2g_interfaces.F90:39-44 */
typedef struct {
    int Nx, Ny, Nz;
    double dx, dy;
    void *z;             /* Nz+1 real(8) cell borders */
    void *dz;            /* Nz real(8) cell thicknesses */
} GIEM2G_ANOMALY_TYPE;

/* giem2g_interfaces.F90:46-58 */
typedef struct {
    long long tensor_size;
    long long ie_kernel_buffer_length;
    long long fft_buffers_length;
    long long comm64;
    void *giem2g_tensor;  /* out of giem2g_calc_data_sizes: the operator handle */
    void *dz;
    void *sqsigb;
    void *csigb;
    void *kernel_buffer;
    void *fft_buffer_in;
    void *fft_buffer_out;
} GIEM2G_DATA_TYPE;

/* ---- reference entry points --------------------------------------------- */
/* giem2g_interfaces.F90:76-100  sizes + allocation of the operator handle */
void giem2g_calc_data_sizes(GIEM2G_ANOMALY_TYPE anomaly, GIEM2G_DATA_TYPE *data);
/* giem2g_interfaces.F90:102-141 geometry, device buffers */
void giem2g_prepare_ie_kernel(GIEM2G_ANOMALY_TYPE anomaly, GIEM2G_DATA_TYPE data);
/* giem2g_interfaces.F90:144-174 spatial Green's tensor for angular frequency omega (FP64, GPU) */
void giem2g_calc_ie_kernel(void *ie, GIEM2G_BACKGROUND_TYPE bkg, GIEM2G_ANOMALY_TYPE anomaly, double omega);
/* giem2g_interfaces.F90:176-188 spectral transform of the tensor (FP64, GPU) */
void giem2g_calc_fft_of_ie_kernel(void *ie);
/* giem2g_interfaces.F90:190-201 csiga: Nx*Ny*Nz complex(8), x fastest */
void giem2g_set_anomaly_conductivity(void *ie, void *csiga);
/* giem2g_interfaces.F90:203-232 out = A in, host arrays of 3*Nx*Ny*Nz complex(8) */
void giem2g_apply_ie_operator(void *ie, void *in, void *out);
/* giem2g_interfaces.F90:234-238 */
void giem2g_set_logger(void (*logger)(const char *));
/* giem2g_interfaces.F90:240-247 */
void giem2g_print_stats(void *ie);
/* giem2g_interfaces.F90:248-254 (this implementation also frees the handle) */
void giem2g_delete_ie_operator(void *ie);

/* ---- status ---------------------------------------------------------------- */
int giem2g_last_status(void);
const char *giem2g_last_error(void);
/* Cumulative number of kernels this library has launched (all operators, this process). */
long long giem2g_kernel_launch_count(void);

/* ---- extensions -------------------------------------------------------------- */
/* Background only (PreparePreconditioner, calc_ie_tensor_module.F90:295-306):
 * layer numbers, per-cell csigb and sqrt(Re csigb), without computing the tensor. */
int giem2g_set_background(void *ie, GIEM2G_BACKGROUND_TYPE bkg, double omega);
/* Upload / download the FP64 spatial tensor.  symm: [Nx][Ny][4][Nz(Nz+1)/2] packed upper
 * (xx,xy,yy,zz), asym: [Nx][Ny][2][Nz*Nz] column-major (xz,yz) -- the reference's
 * G_symm / G_asym of calc_ie_tensor_module.F90:278-288 with all ly on one process. */
int giem2g_set_ie_kernel_spatial(void *ie, const void *symm, const void *asym);
int giem2g_get_ie_kernel_spatial(void *ie, void *symm, void *asym);
/* Download the spectral tensor in the same shapes, indexed [kx-pair][ky] (G_symmT/G_asymT). */
int giem2g_get_ie_kernel_spectral(void *ie, void *symm_hat, void *asym_hat);
/* Device-pointer apply on the operator's stream.  precision 0: complex128 vectors and
 * FP64 tensor; precision 1: complex64 vectors and tensor (FP32 accumulation). */
int giem2g_apply_ie_operator_device(void *ie, const void *d_in, void *d_out, int precision);
/* No counterpart in the reference.  The same apply as giem2g_apply_ie_operator_device, but it
 * allocates nothing: the apply's intermediates live in one static device array of the library
 * (32 MiB per device, shared by every call and operator on that device) instead of the operator's
 * buffers.  For hosts that must not allocate device memory after start-up.  Grids that need more
 * than 32 MiB of intermediates (18*Nx*Ny*Nz complex of the precision) are rejected with status
 * -1 and a message.  The first call on a device sets up the array's address; make it before any stream
 * capture on that device (and again after a device reset, which repeats the set-up).  Calls that overlap
 * on the GPU race on the shared array: each operator has its own stream, so calls on two operators of one
 * device must be ordered by the host (an event or a synchronisation) even when one thread issues them. */
int giem2g_apply_ie_operator_device_static(void *ie, const void *d_in, void *d_out, int precision);
/* Synchronise the operator's stream and report a device-side error word (bounded waits that ran
 * out) as a nonzero status. */
int giem2g_check_device_error(void *ie);
/* Contraction tile-shape variants available for a precision (0 or 1) at this Nz, and selection of one
 * (what the autotuner in giem2g_b200.autotune sets after timing them). */
int giem2g_contract_variants(void *ie, int precision);  /* precision 2: paired complex64 */
int giem2g_set_contract_variant(void *ie, int precision, int variant);
/* Lines per CTA of the FFT passes (4, 8, 16 or 32; default 32), also set by the autotuner: for both
 * precisions, or for one (0 complex128, 1 complex64, the paired apply included). */
int giem2g_set_fft_lines(void *ie, int lines);
int giem2g_set_fft_lines_precision(void *ie, int precision, int lines);
/* Kernel timing: with on != 0, every device apply outside a stream capture records CUDA events around
 * its contraction launch; giem2g_last_contract_ms returns the last one (ms, -1 if none). */
int giem2g_set_kernel_timing(void *ie, int on);
double giem2g_last_contract_ms(void *ie);
/* CUDA stream the operator's kernels run on (cudaStream_t).  It is created non-blocking, so it does
 * not wait for the legacy default stream: every call that takes device pointers is ordered after
 * earlier work on this stream only.  A caller whose inputs come from another stream makes this stream
 * wait for them (cudaStreamWaitEvent) before the call, and makes its consumers wait for this stream
 * after it (the Python layer, giem2g_b200, does both against torch's current stream). */
void *giem2g_get_stream(void *ie);
/* Milliseconds of device time of the last device apply (CUDA events), and kernels it launched. */
double giem2g_last_apply_ms(void *ie);
int giem2g_last_kernel_launches(void *ie);
/* Operator applies since creation or the last giem2g_print_stats (its "Number of matrix-vector
 * multiplications", Integral_Equation_Module.F90:473-484): every apply entry point and solve counts. */
long long giem2g_apply_count(void *ie);

/* FGMRES_CTL_TYPE (data_types_module.F90:49-55) */
typedef struct {
    double misfit;       /* outer tolerance */
    int fgmres_maxit;    /* MaxRestart */
    int gmres_buf;       /* InnerBufferSize */
    int fgmres_buf;      /* OuterBufferSize */
    int precision;       /* 0 plain FP64; 1 mixed: complex64 inner GMRES, FP64 outer;
                            -1: the operator's mode (giem2g_set_precision) */
} GIEM2G_FGMRES_CTL;

/* The operator's precision mode (default 0).  Mode 1 makes the reference-facing apply
 * giem2g_apply_ie_operator compute in complex64 (its vectors stay complex(8)) and is the precision of
 * solves and batches whose control block says -1.  No counterpart in the reference (FP64 only). */
int giem2g_set_precision(void *ie, int mode);

/* RESULT_INFO (GFGMRES/fgmres_interfaces.F90:34-39) + counters */
typedef struct {
    int iterations;
    double bea;          /* Arnoldi misfit */
    double be;           /* true misfit */
    int stat;            /* 1 CONVERGED, 2 NON_TRUE_CONVERGED, -1 NON_CONVERGED, -3 INTERUPTED */
    int applies_fp64;
    int applies_fp32;
    double device_ms;
    int precond_steps;   /* outer steps preconditioned through the outer preconditioner hook */
} GIEM2G_RESULT;

/* SolveEquation (ie_solver_module.F90:43-114): E_bkg, Esol, E0 host arrays (Nx,Ny,Nz,3)
 * complex(8); E0 may be NULL (guess = sqrt(Re sigma_b) * E_bkg).  Esol receives a*chi. */
int giem2g_solve(void *ie, const void *E_bkg, void *Esol, const void *E0, GIEM2G_FGMRES_CTL ctl,
                 GIEM2G_RESULT *info);
/* Same with device pointers (complex128), on the operator's stream. */
int giem2g_solve_device(void *ie, const void *d_E_bkg, void *d_Esol, const void *d_E0, GIEM2G_FGMRES_CTL ctl,
                        GIEM2G_RESULT *info);
/* Outer Arnoldi misfit after each outer iteration of the last solve; returns the count copied. */
int giem2g_get_misfit_history(void *ie, double *out, int max_len);
/* Outer right preconditioner hook: the slot that SET_RIGHT_PRECONDTIONER (seq_fgmres.F90:92-102) fills
 * with the inner GMRES in the reference, here open to the learned preconditioner.
 * fn(user, d_v, d_z, n, stream) receives V_j (complex128, n elements, device) and writes its guess of
 * A^-1 V_j to d_z (complex128, device) on `stream`, returning 0 (nonzero: the hook is dropped for the
 * rest of the solve).  mode 1: the guess starts the inner GMRES cycle (x0 = guess instead of x0 = V_j);
 * mode 2: the guess is Z_j itself (no inner cycle); mode 0 removes the hook.  Whenever an outer step
 * through the hook fails to halve the Arnoldi misfit, the plain inner GMRES takes over for the rest of
 * the solve.  Single-instance solves only (giem2g_solve, giem2g_solve_device). */
typedef int (*giem2g_precond_fn)(void *user, const void *d_v, void *d_z, long long n, void *stream);
int giem2g_set_outer_preconditioner(void *ie, int mode, giem2g_precond_fn fn, void *user);
/* The learned preconditioner in that slot without a host-side network: kind 0 = plain inner GMRES
 * (removes it), 1 = the network's guess starts the inner GMRES cycle, 2 = the guess replaces the inner
 * cycle (with the fallback rule above).  weights_path: the .npz of giem2g_b200/weights (float32 [Cout][Kp]
 * matrices of the 12 convolutions); the network reads log10 of the operator's anomaly conductivity (set
 * it first) and its frequency.  Nx, Ny, Nz must be multiples of 8.  No counterpart in the reference. */
int giem2g_set_preconditioner(void *ie, int kind, const char *weights_path);
/* network evaluations since giem2g_set_preconditioner */
long long giem2g_preconditioner_calls(void *ie);
/* the registered network once, outside a solve: d_z = d_v + rms(d_v) * net(d_v) (complex128, device,
 * 3*Nx*Ny*Nz elements, on the operator's stream; synchronises) */
int giem2g_apply_preconditioner(void *ie, const void *d_v, void *d_z);

/* ---- batched solves -----------------------------------------------------------
 * The reference solves one (frequency, polarisation) after another (giem2g.F90:336-373).  A batch
 * holds n instances, each an operator handle (one per frequency, already through
 * giem2g_calc_fft_of_ie_kernel and giem2g_set_anomaly_conductivity); the same handle may appear
 * twice in a row for the two polarisations of one frequency.  A batched solve runs every instance's
 * nested FGMRES in lockstep on ies[0]'s stream: one captured inner cycle serves all instances, and
 * in mixed precision consecutive instances of one operator share every tensor read.  Each instance
 * keeps its own iterates, misfit history and status; converged instances are masked off.  The
 * buffer sizes and precision of ctl are fixed at creation.  Returns NULL on error. */
void *giem2g_batch_create(void *const *ies, int n, GIEM2G_FGMRES_CTL ctl);
/* device vectors: d_E_bkg[i], d_Esol[i] complex128 of instance i's size; d_E0 (or d_E0[i]) may be NULL */
int giem2g_batch_solve_device(void *batch, const void *const *d_E_bkg, void *const *d_Esol,
                              const void *const *d_E0, GIEM2G_FGMRES_CTL ctl, GIEM2G_RESULT *info);
/* the same with host arrays (copied in and out every call) */
int giem2g_solve_batched(void *batch, const void *const *E_bkg, void *const *Esol, const void *const *E0,
                         GIEM2G_FGMRES_CTL ctl, GIEM2G_RESULT *info);
int giem2g_batch_misfit_history(void *batch, int i, double *out, int max_len);
void giem2g_batch_delete(void *batch);
/* nv device vectors through one operator; precision 1 applies them two at a time with shared tensor
 * reads, precision 0 one at a time. */
int giem2g_apply_ie_operator_device_batch(void *ie, int nv, const void *const *d_in, void *const *d_out,
                                          int precision);

/* ---- learned preconditioner building blocks (no counterpart in the reference) ----------------
 * BF16 GEMM on the tcgen05 tensor cores with FP32 accumulation and output:
 * C[M][N] = A[M][K] B[N][K]^T (accumulate 0) or C += A B^T (accumulate 1); A, B row-major bf16 with
 * K contiguous; K, lda, ldb multiples of 8.  d_err: device int set nonzero if a bounded wait gave up
 * (NULL: an internal one).  stream: cudaStream_t or NULL. */
int giem2g_gemm_bf16_tn(const void *A, const void *B, float *C, int M, int N, int K, int lda, int ldb, int ldc,
                        int accumulate, int *d_err, void *stream);
/* 3x3x3 convolution with padding 1 and stride 1 or 2 on channels-last volumes x[N][D][H][W][C] (bf16):
 * cols[N*Do*Ho*Wo][Kp] with column tap*C + c, tap = (dz*3 + dy)*3 + dx, zero beyond 27C (Kp >= 27C,
 * multiple of 8); col2im is its adjoint, dx[N][D][H][W][C] (fp32) = sum of dcols over the taps that
 * read each input element. */
int giem2g_im2col3d_bf16(const void *x, void *cols, int N, int D, int H, int W, int C, int stride, int Kp,
                         void *stream);
int giem2g_col2im3d_f32(const float *dcols, float *dx, int N, int D, int H, int W, int C, int stride, int Kp,
                        void *stream);

/* ---- receiver continuation ---------------------------------------------------------------------
 * Fields at receiver points from the currents j = (csiga - csigb) E of an IE solution.  The reference
 * has no C interface for this part; these entry points follow its Fortran module routines:
 *   giem2g_rc_create             PrepareRecvs (data_types_module.F90:124-152) +
 *                                PrepareContinuationOperator (Continuation_Function_Module.F90:84-164)
 *   giem2g_rc_calc_kernel        CalcRecalculationGreenTensor (calc_rc_tensor_module.F90:38-229)
 *   giem2g_rc_calc_fft_of_kernel CalcFFTofRCTensor (Continuation_Function_Module.F90:330-366)
 *   giem2g_rc_set_anomaly_conductivity  FinalizeRCOperator (:165-196)
 *   giem2g_rc_recalculate        ReCalculation (:198-239): E and H at the receivers, anomalous part
 *   giem2g_rc_delete             DeleteRC_OP (:371-380)
 * Receivers sit on the anomaly's lateral grid: receiver r at cell (ix, iy) is the point
 * ((ix+1/2) dx + x_shift[r], (iy+1/2) dy + y_shift[r], zrecv[r]).  A receiver depth strictly inside an
 * anomaly cell is moved to the cell's top border, as PrepareRecvs does; giem2g_rc_receivers reports the
 * depths used, each receiver's layer and the number of anomaly cells above it.
 * Fields: E [3][Nz][Ny][Nx] as the IE vectors (Fortran E(Nx,Ny,Nz,3)); Ea, Ha complex(8)
 * [Ny][Nx][3][Nr] (Fortran Ea(Nr,3,Nx,Ny), the reference's layout).  The total fields add the normal
 * field of the layered background at the receiver depths (sources_module.F90:26-66).
 * FP64 throughout.  Nx and Ny powers of two (2*Nx, 2*Ny <= 2048), Nz <= 64, up to 16 layers. */
void *giem2g_rc_create(GIEM2G_BACKGROUND_TYPE bkg, GIEM2G_ANOMALY_TYPE anomaly, int Nr, const double *zrecv,
                       const double *x_shift, const double *y_shift);
int giem2g_rc_receivers(void *rc, double *zrecv, int *recv_layer, int *anom_cell);
/* bkg.csigb: complex conductivities at the frequency (air first); omega = 2 pi f */
int giem2g_rc_calc_kernel(void *rc, GIEM2G_BACKGROUND_TYPE bkg, double omega);
int giem2g_rc_calc_fft_of_kernel(void *rc);
/* the current tensor (spatial after giem2g_rc_calc_kernel, spectral after giem2g_rc_calc_fft_of_kernel):
 * complex(8) [2Ny][2Nx][15][Nr][Nz]; lag index ix < Nx is lag ix, ix > Nx is ix - 2Nx, ix = Nx is zero
 * (same in y); components E xx xy xz yy yz zx zy zz, H xx xy xz yx yz zx zy (const_module.F90:112-130) */
int giem2g_rc_get_kernel(void *rc, void *G);
/* csiga complex(8) (Nx,Ny,Nz), x fastest, at the frequency of the kernel (copied) */
int giem2g_rc_set_anomaly_conductivity(void *rc, const void *csiga);
int giem2g_rc_recalculate(void *rc, const void *E, void *Ea, void *Ha);
/* the same with device buffers, on giem2g_rc_get_stream(rc) */
int giem2g_rc_recalculate_device(void *rc, const void *d_E, void *d_Ea, void *d_Ha);
void *giem2g_rc_get_stream(void *rc);
void giem2g_rc_delete(void *rc);

/* Failure-detection self-test (no counterpart in the reference): runs the library's bounded wait on an
 * mbarrier that nothing completes, with a limit of limit_ms (1..2000); returns the device error code the
 * wait recorded (77) after about limit_ms, or a negative status.  The context stays usable. */
int giem2g_selftest_bounded_wait(int limit_ms);

#ifdef __cplusplus
}
#endif
#endif
