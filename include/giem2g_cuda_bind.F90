! giem2g_cuda_bind.F90 -- Fortran 2003 ISO_C_BINDING interface to libgiem2g_b200 (include/giem2g.h).
!
! The reference's Fortran host (giem2g.F90) keeps its driver, JSON input, background set-up, plane-wave
! source and output.  Two subroutine bodies route to this module:
!   APPLY_PRECOND (apply_ie_operator_module.F90:39)  -> giem2g_apply_ie_operator
!   SolveEquation (ie_solver_module.F90:43)          -> giem2g_cuda_solve_equation (below)
! and the per-frequency set-up of the operator (giem2g_interfaces.F90:76-188, the extrEMe host sequence)
! becomes giem2g_calc_data_sizes + giem2g_prepare_ie_kernel once per anomaly, then
! giem2g_calc_ie_kernel + giem2g_calc_fft_of_ie_kernel + giem2g_set_anomaly_conductivity per frequency.
!
! Derived types mirror the C structs field by field (BIND(C) layout).  Vectors are COMPLEX(C_DOUBLE_COMPLEX)
! arrays (Nx, Ny, Nz, 3), x fastest, passed with C_LOC.  Every extension returns 0 or a negative status
! (-1 argument, -2 CUDA, -3 state, -4 unsupported, -5 numeric, -6 out of memory); the nine reference entry
! points return nothing and record their status in giem2g_last_status().
MODULE giem2g_cuda_bind
  USE, INTRINSIC :: ISO_C_BINDING
  IMPLICIT NONE
  PRIVATE :: c_string_to_fortran

  ! giem2g_interfaces.F90:33-37
  TYPE, BIND(C) :: GIEM2G_BACKGROUND_TYPE
     INTEGER(C_INT) :: Nl
     TYPE(C_PTR)    :: csigb
     TYPE(C_PTR)    :: thickness
  END TYPE GIEM2G_BACKGROUND_TYPE

  ! giem2g_interfaces.F90:39-44
  TYPE, BIND(C) :: GIEM2G_ANOMALY_TYPE
     INTEGER(C_INT) :: Nx, Ny, Nz
     REAL(C_DOUBLE) :: dx, dy
     TYPE(C_PTR)    :: z
     TYPE(C_PTR)    :: dz
  END TYPE GIEM2G_ANOMALY_TYPE

  ! giem2g_interfaces.F90:46-58
  TYPE, BIND(C) :: GIEM2G_DATA_TYPE
     INTEGER(C_LONG_LONG) :: tensor_size, ie_kernel_buffer_length, fft_buffers_length, comm64
     TYPE(C_PTR) :: giem2g_tensor, dz, sqsigb, csigb, kernel_buffer, fft_buffer_in, fft_buffer_out
  END TYPE GIEM2G_DATA_TYPE

  ! FGMRES_CTL_TYPE (data_types_module.F90:49-55) + precision (0 FP64, 1 mixed, -1 the operator's mode)
  TYPE, BIND(C) :: GIEM2G_FGMRES_CTL
     REAL(C_DOUBLE) :: misfit
     INTEGER(C_INT) :: fgmres_maxit, gmres_buf, fgmres_buf, precision
  END TYPE GIEM2G_FGMRES_CTL

  ! RESULT_INFO (GFGMRES/fgmres_interfaces.F90:34-39) + counters
  TYPE, BIND(C) :: GIEM2G_RESULT
     INTEGER(C_INT) :: iterations
     REAL(C_DOUBLE) :: bea, be
     INTEGER(C_INT) :: stat, applies_fp64, applies_fp32
     REAL(C_DOUBLE) :: device_ms
     INTEGER(C_INT) :: precond_steps
  END TYPE GIEM2G_RESULT

  INTERFACE
     ! ---- the reference's C interface (giem2g_interfaces.F90:76-254) ----
     SUBROUTINE giem2g_calc_data_sizes(anomaly, data) BIND(C, NAME='giem2g_calc_data_sizes')
       IMPORT :: GIEM2G_ANOMALY_TYPE, GIEM2G_DATA_TYPE
       TYPE(GIEM2G_ANOMALY_TYPE), VALUE :: anomaly
       TYPE(GIEM2G_DATA_TYPE) :: data
     END SUBROUTINE giem2g_calc_data_sizes

     SUBROUTINE giem2g_prepare_ie_kernel(anomaly, data) BIND(C, NAME='giem2g_prepare_ie_kernel')
       IMPORT :: GIEM2G_ANOMALY_TYPE, GIEM2G_DATA_TYPE
       TYPE(GIEM2G_ANOMALY_TYPE), VALUE :: anomaly
       TYPE(GIEM2G_DATA_TYPE), VALUE :: data
     END SUBROUTINE giem2g_prepare_ie_kernel

     SUBROUTINE giem2g_calc_ie_kernel(ie, bkg, anomaly, omega) BIND(C, NAME='giem2g_calc_ie_kernel')
       IMPORT :: C_PTR, C_DOUBLE, GIEM2G_BACKGROUND_TYPE, GIEM2G_ANOMALY_TYPE
       TYPE(C_PTR), VALUE :: ie
       TYPE(GIEM2G_BACKGROUND_TYPE), VALUE :: bkg
       TYPE(GIEM2G_ANOMALY_TYPE), VALUE :: anomaly
       REAL(C_DOUBLE), VALUE :: omega
     END SUBROUTINE giem2g_calc_ie_kernel

     SUBROUTINE giem2g_calc_fft_of_ie_kernel(ie) BIND(C, NAME='giem2g_calc_fft_of_ie_kernel')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ie
     END SUBROUTINE giem2g_calc_fft_of_ie_kernel

     SUBROUTINE giem2g_set_anomaly_conductivity(ie, csiga) BIND(C, NAME='giem2g_set_anomaly_conductivity')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ie, csiga
     END SUBROUTINE giem2g_set_anomaly_conductivity

     SUBROUTINE giem2g_apply_ie_operator(ie, v_in, v_out) BIND(C, NAME='giem2g_apply_ie_operator')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ie, v_in, v_out
     END SUBROUTINE giem2g_apply_ie_operator

     SUBROUTINE giem2g_set_logger(logger) BIND(C, NAME='giem2g_set_logger')
       IMPORT :: C_FUNPTR
       TYPE(C_FUNPTR), VALUE :: logger
     END SUBROUTINE giem2g_set_logger

     SUBROUTINE giem2g_print_stats(ie) BIND(C, NAME='giem2g_print_stats')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ie
     END SUBROUTINE giem2g_print_stats

     SUBROUTINE giem2g_delete_ie_operator(ie) BIND(C, NAME='giem2g_delete_ie_operator')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: ie
     END SUBROUTINE giem2g_delete_ie_operator

     ! ---- status ----
     INTEGER(C_INT) FUNCTION giem2g_last_status() BIND(C, NAME='giem2g_last_status')
       IMPORT :: C_INT
     END FUNCTION giem2g_last_status

     TYPE(C_PTR) FUNCTION giem2g_last_error() BIND(C, NAME='giem2g_last_error')
       IMPORT :: C_PTR
     END FUNCTION giem2g_last_error

     ! ---- extensions used by the replaced bodies ----
     INTEGER(C_INT) FUNCTION giem2g_set_precision(ie, mode) BIND(C, NAME='giem2g_set_precision')
       IMPORT :: C_PTR, C_INT
       TYPE(C_PTR), VALUE :: ie
       INTEGER(C_INT), VALUE :: mode
     END FUNCTION giem2g_set_precision

     INTEGER(C_INT) FUNCTION giem2g_solve(ie, E_bkg, Esol, E0, ctl, info) BIND(C, NAME='giem2g_solve')
       IMPORT :: C_PTR, C_INT, GIEM2G_FGMRES_CTL, GIEM2G_RESULT
       TYPE(C_PTR), VALUE :: ie, E_bkg, Esol, E0
       TYPE(GIEM2G_FGMRES_CTL), VALUE :: ctl
       TYPE(GIEM2G_RESULT) :: info
     END FUNCTION giem2g_solve

     INTEGER(C_INT) FUNCTION giem2g_get_misfit_history(ie, out, max_len) BIND(C, NAME='giem2g_get_misfit_history')
       IMPORT :: C_PTR, C_INT, C_DOUBLE
       TYPE(C_PTR), VALUE :: ie
       REAL(C_DOUBLE) :: out(*)
       INTEGER(C_INT), VALUE :: max_len
     END FUNCTION giem2g_get_misfit_history

     ! batches: ies, E_bkg, Esol and E0 are arrays of n C pointers (E0 may be C_NULL_PTR)
     TYPE(C_PTR) FUNCTION giem2g_batch_create(ies, n, ctl) BIND(C, NAME='giem2g_batch_create')
       IMPORT :: C_PTR, C_INT, GIEM2G_FGMRES_CTL
       TYPE(C_PTR) :: ies(*)
       INTEGER(C_INT), VALUE :: n
       TYPE(GIEM2G_FGMRES_CTL), VALUE :: ctl
     END FUNCTION giem2g_batch_create

     INTEGER(C_INT) FUNCTION giem2g_solve_batched(batch, E_bkg, Esol, E0, ctl, info) &
          BIND(C, NAME='giem2g_solve_batched')
       IMPORT :: C_PTR, C_INT, GIEM2G_FGMRES_CTL, GIEM2G_RESULT
       TYPE(C_PTR), VALUE :: batch
       TYPE(C_PTR) :: E_bkg(*), Esol(*)
       TYPE(C_PTR), VALUE :: E0
       TYPE(GIEM2G_FGMRES_CTL), VALUE :: ctl
       TYPE(GIEM2G_RESULT) :: info(*)
     END FUNCTION giem2g_solve_batched

     SUBROUTINE giem2g_batch_delete(batch) BIND(C, NAME='giem2g_batch_delete')
       IMPORT :: C_PTR
       TYPE(C_PTR), VALUE :: batch
     END SUBROUTINE giem2g_batch_delete

     INTEGER(C_SIZE_T) FUNCTION c_strlen(s) BIND(C, NAME='strlen')
       IMPORT :: C_PTR, C_SIZE_T
       TYPE(C_PTR), VALUE :: s
     END FUNCTION c_strlen
  END INTERFACE

CONTAINS

  ! The library's last error message as a Fortran string (for STOP and log lines).
  FUNCTION giem2g_error_message() RESULT(msg)
    CHARACTER(LEN=:), ALLOCATABLE :: msg
    msg = c_string_to_fortran(giem2g_last_error())
  END FUNCTION giem2g_error_message

  FUNCTION c_string_to_fortran(p) RESULT(s)
    TYPE(C_PTR), INTENT(IN) :: p
    CHARACTER(LEN=:), ALLOCATABLE :: s
    CHARACTER(KIND=C_CHAR), POINTER :: chars(:)
    INTEGER :: i, n
    IF (.NOT. C_ASSOCIATED(p)) THEN
       s = ''
       RETURN
    END IF
    n = INT(c_strlen(p))
    CALL C_F_POINTER(p, chars, [n])
    ALLOCATE(CHARACTER(LEN=n) :: s)
    DO i = 1, n
       s(i:i) = chars(i)
    END DO
  END FUNCTION c_string_to_fortran

  ! The body SolveEquation (ie_solver_module.F90:43-114) routes to: the nested FGMRES of
  ! GIEM2G_FGMRES (:141-258) on the GPU.  E_bkg, Esol and the optional initial guess E0 are the
  ! caller's (Nx,Ny,Nz,3) complex(8) arrays; misfit, max_restart, inner_buf and outer_buf are the
  ! FGMRES_CTL_TYPE fields (Tolerance, MaxRestart, InnerBufferSize, OuterBufferSize); precision 0 is the
  ! reference's FP64 solve, 1 the mixed one.  Returns the status and fills info.
  FUNCTION giem2g_cuda_solve_equation(gpu, misfit, max_restart, inner_buf, outer_buf, precision, &
                                      E_bkg, Esol, info, E0) RESULT(status)
    TYPE(C_PTR), INTENT(IN) :: gpu
    REAL(C_DOUBLE), INTENT(IN) :: misfit
    INTEGER, INTENT(IN) :: max_restart, inner_buf, outer_buf, precision
    COMPLEX(C_DOUBLE_COMPLEX), TARGET, INTENT(IN) :: E_bkg(:, :, :, :)
    COMPLEX(C_DOUBLE_COMPLEX), TARGET, INTENT(INOUT) :: Esol(:, :, :, :)
    TYPE(GIEM2G_RESULT), INTENT(OUT) :: info
    COMPLEX(C_DOUBLE_COMPLEX), TARGET, INTENT(IN), OPTIONAL :: E0(:, :, :, :)
    INTEGER :: status
    TYPE(GIEM2G_FGMRES_CTL) :: ctl
    TYPE(C_PTR) :: guess
    ctl%misfit = misfit
    ctl%fgmres_maxit = INT(max_restart, C_INT)
    ctl%gmres_buf = INT(inner_buf, C_INT)
    ctl%fgmres_buf = INT(outer_buf, C_INT)
    ctl%precision = INT(precision, C_INT)
    guess = C_NULL_PTR
    IF (PRESENT(E0)) guess = C_LOC(E0)
    status = INT(giem2g_solve(gpu, C_LOC(E_bkg), C_LOC(Esol), guess, ctl, info))
  END FUNCTION giem2g_cuda_solve_equation

END MODULE giem2g_cuda_bind
