!
! fft_parallele_gpu -- drop-in for the dealiased products of MODULE fft_parallele
! (SOURCES/POST_PROCESSING/fft_parallel.F90) backed by the B200 library
! libsfemans_nl.so through ISO_C_BINDING.
!
! Same PUBLIC names, argument lists and argument meaning as
!   FFT_PAR_CROSS_PROD_DCL  fft_parallel.F90:147
!   FFT_PAR_DOT_PROD_DCL    fft_parallel.F90:330
!   FFT_PAR_PROD_DCL        fft_parallel.F90:502
!   FFT_PAR_DIV_DCL         fft_parallel.F90:667
!   FFT_SCALAR_VECT_DCL     fft_parallel.F90:1021
!   FFT_TENSOR_DCL          fft_parallel.F90:1543
!   FFT_PAR_REAL            fft_parallel.F90:28    (V_out ALLOCATABLE, allocated here as in the reference)
!   FFT_MAX_VEL_DCL         fft_parallel.F90:1426
! With one Fourier rank (nb_procs == 1) the library holds every mode and
! bloc_size is only checked (np <= nb_procs*bloc_size).  With nb_procs > 1
! the products keep the reference's exchange (fft_parallel.F90:205-217 and
! :306-324): the library lays out the send buffers, MPI_ALLTOALL gathers the
! rank's block of bloc_size points with all modes, the library computes the
! block's product on the GPU, a second MPI_ALLTOALL returns every rank its
! modes, and the library unpacks them (dummy points dropped).  temps(3), when
! present, is zeroed and receives the exchange and host<->device copy seconds
! in temps(1), the kernel seconds in temps(2) and the buffer layout seconds in
! temps(3).  FFT_PAR_REAL and FFT_MAX_VEL_DCL run on one rank.  A non-zero status
! from the library prints 'BUG in FFT_PAR_...' with the library's message and
! STOPs, as the reference does (fft_parallel.F90:188-191).
!
MODULE fft_parallele_gpu
#include "petsc/finclude/petsc.h"
  USE petsc
  USE ISO_C_BINDING
  IMPLICIT NONE
  PRIVATE
  PUBLIC :: FFT_PAR_CROSS_PROD_DCL, FFT_PAR_DOT_PROD_DCL, FFT_PAR_PROD_DCL
  PUBLIC :: FFT_PAR_DIV_DCL, FFT_SCALAR_VECT_DCL, FFT_TENSOR_DCL
  PUBLIC :: FFT_PAR_REAL, FFT_MAX_VEL_DCL

  INTERFACE
     FUNCTION sfnl_fft_par_cross_prod_dcl(V1_in, V2_in, V_out, np, nb_field, m_max_c, nb_procs, &
          bloc_size, m_max_pad, temps) RESULT(rc) BIND(C, NAME='sfnl_fft_par_cross_prod_dcl')
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: V1_in, V2_in
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: V_out
       INTEGER(C_INT), VALUE :: np, nb_field, m_max_c, nb_procs, bloc_size, m_max_pad
       TYPE(C_PTR), VALUE    :: temps
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_par_cross_prod_dcl

     FUNCTION sfnl_fft_par_dot_prod_dcl(V1_in, V2_in, c_out, np, nb_field, m_max_c, nb_procs, &
          bloc_size, m_max_pad, temps) RESULT(rc) BIND(C, NAME='sfnl_fft_par_dot_prod_dcl')
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: V1_in, V2_in
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: c_out
       INTEGER(C_INT), VALUE :: np, nb_field, m_max_c, nb_procs, bloc_size, m_max_pad
       TYPE(C_PTR), VALUE    :: temps
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_par_dot_prod_dcl

     FUNCTION sfnl_fft_par_prod_dcl(c1_in, c2_in, c_out, np, m_max_c, nb_procs, &
          bloc_size, m_max_pad, temps) RESULT(rc) BIND(C, NAME='sfnl_fft_par_prod_dcl')
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: c1_in, c2_in
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: c_out
       INTEGER(C_INT), VALUE :: np, m_max_c, nb_procs, bloc_size, m_max_pad
       TYPE(C_PTR), VALUE    :: temps
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_par_prod_dcl

     FUNCTION sfnl_fft_par_div_dcl(c1_in, c2_in, c_out, np, m_max_c, nb_procs, &
          bloc_size, m_max_pad, temps) RESULT(rc) BIND(C, NAME='sfnl_fft_par_div_dcl')
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: c1_in, c2_in
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: c_out
       INTEGER(C_INT), VALUE :: np, m_max_c, nb_procs, bloc_size, m_max_pad
       TYPE(C_PTR), VALUE    :: temps
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_par_div_dcl

     FUNCTION sfnl_fft_scalar_vect_dcl(V1_in, V2_in, V_out, pb, np, nb_field1, nb_field2, m_max_c, &
          nb_procs, bloc_size, m_max_pad, temps) RESULT(rc) BIND(C, NAME='sfnl_fft_scalar_vect_dcl')
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: V1_in, V2_in
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: V_out
       INTEGER(C_INT), VALUE :: pb, np, nb_field1, nb_field2, m_max_c, nb_procs, bloc_size, m_max_pad
       TYPE(C_PTR), VALUE    :: temps
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_scalar_vect_dcl

     FUNCTION sfnl_fft_tensor_dcl(V1_in, V2_in, V_out, np, nb_field, m_max_c, nb_procs, &
          bloc_size, m_max_pad, opt_tension, temps) RESULT(rc) BIND(C, NAME='sfnl_fft_tensor_dcl')
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: V1_in, V2_in
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: V_out
       INTEGER(C_INT), VALUE :: np, nb_field, m_max_c, nb_procs, bloc_size, m_max_pad, opt_tension
       TYPE(C_PTR), VALUE    :: temps
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_tensor_dcl

     FUNCTION sfnl_fft_par_real_planes(m_max, opt_nb_plane) RESULT(n) BIND(C, NAME='sfnl_fft_par_real_planes')
       IMPORT :: C_INT
       INTEGER(C_INT), VALUE :: m_max, opt_nb_plane
       INTEGER(C_INT)        :: n
     END FUNCTION sfnl_fft_par_real_planes

     FUNCTION sfnl_fft_par_real(V1_in, V_out, np, nb_field, m_max_c, nb_procs, opt_nb_plane) RESULT(rc) &
          BIND(C, NAME='sfnl_fft_par_real')
       IMPORT :: C_INT, C_DOUBLE
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: V1_in
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: V_out
       INTEGER(C_INT), VALUE :: np, nb_field, m_max_c, nb_procs, opt_nb_plane
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_par_real

     FUNCTION sfnl_fft_max_vel_dcl(V1_in, V_out, np, nb_field, m_max_c, nb_procs, bloc_size, m_max_pad) RESULT(rc) &
          BIND(C, NAME='sfnl_fft_max_vel_dcl')
       IMPORT :: C_INT, C_DOUBLE
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN) :: V1_in
       REAL(C_DOUBLE), INTENT(OUT)              :: V_out
       INTEGER(C_INT), VALUE :: np, nb_field, m_max_c, nb_procs, bloc_size, m_max_pad
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_max_vel_dcl

     FUNCTION sfnl_fft_par_pack_modes(V, send, np, nslot, m_max_c, nb_procs, bloc_size, ew) RESULT(rc) &
          BIND(C, NAME='sfnl_fft_par_pack_modes')
       IMPORT :: C_INT, C_DOUBLE
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: V
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: send
       INTEGER(C_INT), VALUE :: np, nslot, m_max_c, nb_procs, bloc_size, ew
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_par_pack_modes

     FUNCTION sfnl_fft_par_block(op, recv1, recv2, back, bloc_size, m_max_c, nb_procs, m_max_pad, temps) RESULT(rc) &
          BIND(C, NAME='sfnl_fft_par_block')
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       INTEGER(C_INT), VALUE :: op
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: recv1, recv2
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: back
       INTEGER(C_INT), VALUE :: bloc_size, m_max_c, nb_procs, m_max_pad
       TYPE(C_PTR), VALUE    :: temps
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_par_block

     FUNCTION sfnl_fft_par_unpack_modes(got, V_out, np, nslot, m_max_c, nb_procs, bloc_size, ew) RESULT(rc) &
          BIND(C, NAME='sfnl_fft_par_unpack_modes')
       IMPORT :: C_INT, C_DOUBLE
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: got
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: V_out
       INTEGER(C_INT), VALUE :: np, nslot, m_max_c, nb_procs, bloc_size, ew
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_fft_par_unpack_modes

     FUNCTION sfnl_last_error() RESULT(msg) BIND(C, NAME='sfnl_last_error')
       IMPORT :: C_PTR
       TYPE(C_PTR) :: msg
     END FUNCTION sfnl_last_error
  END INTERFACE

CONTAINS

  SUBROUTINE check_comm(communicator, nb_procs, what)
    MPI_Comm,         INTENT(IN) :: communicator
    INTEGER,          INTENT(IN) :: nb_procs
    CHARACTER(LEN=*), INTENT(IN) :: what
    INTEGER :: nproc, code
    CALL MPI_COMM_SIZE(communicator, nproc, code)
    IF (nproc /= nb_procs .OR. nb_procs /= 1) THEN
       WRITE(*,*) ' BUG in ', what, ': the GPU path holds all Fourier modes on one rank (nb_procs must be 1)'
       STOP
    END IF
  END SUBROUTINE check_comm

  ! .TRUE. when the products run mode-distributed (nb_procs > 1); the communicator must have nb_procs ranks.
  LOGICAL FUNCTION distributed(communicator, nb_procs, what)
    MPI_Comm,         INTENT(IN) :: communicator
    INTEGER,          INTENT(IN) :: nb_procs
    CHARACTER(LEN=*), INTENT(IN) :: what
    INTEGER :: nproc, code
    CALL MPI_COMM_SIZE(communicator, nproc, code)
    IF (nproc /= nb_procs) THEN
       WRITE(*,*) ' BUG in ', what, ': nb_procs differs from the size of the communicator'
       STOP
    END IF
    distributed = nb_procs > 1
  END FUNCTION distributed

  ! The body of a product routine on a mode-distributed communicator: library op code op (SFNL_OP_*),
  ! inputs of nsl1 and nsl2 slots, output of nout slots (ew = 3 for the tensor's V_out(3, np, 6, m)).
  SUBROUTINE mode_distributed(communicator, op, V1_in, nsl1, V2_in, nsl2, V_out, nout, ew, np, m_max_c, &
       nb_procs, bloc_size, m_max_pad, what, temps)
    MPI_Comm :: communicator
    INTEGER, INTENT(IN) :: op, nsl1, nsl2, nout, ew, np, m_max_c, nb_procs, bloc_size, m_max_pad
    REAL(KIND=8), DIMENSION(*), INTENT(IN)  :: V1_in, V2_in
    REAL(KIND=8), DIMENSION(*), INTENT(OUT) :: V_out
    CHARACTER(LEN=*), INTENT(IN) :: what
    REAL(KIND=8), DIMENSION(:), OPTIONAL, INTENT(INOUT) :: temps
    REAL(KIND=8), DIMENSION(:), ALLOCATABLE :: s1, s2, r1, r2, back, got
    REAL(C_DOUBLE), DIMENSION(3), TARGET :: t3
    REAL(KIND=8) :: t, tcomm, tpack
    INTEGER :: n1, n2, no, code
    INTEGER(C_INT) :: rc
    n1 = bloc_size*nsl1*m_max_c
    n2 = bloc_size*nsl2*m_max_c
    no = bloc_size*nout*m_max_c*ew
    ALLOCATE(s1(n1*nb_procs), r1(n1*nb_procs), s2(n2*nb_procs), r2(n2*nb_procs), back(no*nb_procs), got(no*nb_procs))
    t = MPI_WTIME()
    rc = sfnl_fft_par_pack_modes(V1_in, s1, INT(np, C_INT), INT(nsl1, C_INT), INT(m_max_c, C_INT), &
         INT(nb_procs, C_INT), INT(bloc_size, C_INT), 1_C_INT)
    CALL stop_on_error(rc, what)
    rc = sfnl_fft_par_pack_modes(V2_in, s2, INT(np, C_INT), INT(nsl2, C_INT), INT(m_max_c, C_INT), &
         INT(nb_procs, C_INT), INT(bloc_size, C_INT), 1_C_INT)
    CALL stop_on_error(rc, what)
    tpack = MPI_WTIME() - t
    t = MPI_WTIME()
    CALL MPI_ALLTOALL(s1, n1, MPI_DOUBLE_PRECISION, r1, n1, MPI_DOUBLE_PRECISION, communicator, code)
    CALL MPI_ALLTOALL(s2, n2, MPI_DOUBLE_PRECISION, r2, n2, MPI_DOUBLE_PRECISION, communicator, code)
    tcomm = MPI_WTIME() - t
    rc = sfnl_fft_par_block(INT(op, C_INT), r1, r2, back, INT(bloc_size, C_INT), INT(m_max_c, C_INT), &
         INT(nb_procs, C_INT), INT(m_max_pad, C_INT), C_LOC(t3))
    CALL stop_on_error(rc, what)
    t = MPI_WTIME()
    CALL MPI_ALLTOALL(back, no, MPI_DOUBLE_PRECISION, got, no, MPI_DOUBLE_PRECISION, communicator, code)
    tcomm = tcomm + MPI_WTIME() - t
    t = MPI_WTIME()
    rc = sfnl_fft_par_unpack_modes(got, V_out, INT(np, C_INT), INT(nout, C_INT), INT(m_max_c, C_INT), &
         INT(nb_procs, C_INT), INT(bloc_size, C_INT), INT(ew, C_INT))
    CALL stop_on_error(rc, what)
    tpack = tpack + MPI_WTIME() - t
    DEALLOCATE(s1, r1, s2, r2, back, got)
    IF (PRESENT(temps)) THEN
       temps = 0.d0
       temps(1) = tcomm + t3(1)
       IF (SIZE(temps) > 1) temps(2) = t3(2)
       IF (SIZE(temps) > 2) temps(3) = tpack
    END IF
  END SUBROUTINE mode_distributed

  SUBROUTINE usage_stop(what, why)
    CHARACTER(LEN=*), INTENT(IN) :: what, why
    WRITE(*,*) ' BUG in ', what, ' : ', why
    STOP
  END SUBROUTINE usage_stop

  SUBROUTINE stop_on_error(rc, what)
    INTEGER(C_INT),   INTENT(IN) :: rc
    CHARACTER(LEN=*), INTENT(IN) :: what
    CHARACTER(KIND=C_CHAR), DIMENSION(:), POINTER :: cmsg
    CHARACTER(LEN=256) :: msg
    INTEGER :: i
    IF (rc == 0) RETURN
    CALL C_F_POINTER(sfnl_last_error(), cmsg, [256])
    msg = ' '
    DO i = 1, 256
       IF (cmsg(i) == C_NULL_CHAR) EXIT
       msg(i:i) = cmsg(i)
    END DO
    WRITE(*,*) ' BUG in ', what, ' (status ', rc, '): ', TRIM(msg)
    STOP
  END SUBROUTINE stop_on_error

  SUBROUTINE FFT_PAR_CROSS_PROD_DCL(communicator, V1_in, V2_in, V_out, nb_procs, bloc_size, m_max_pad, temps)
    MPI_Comm :: communicator
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V1_in, V2_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: V_out
    INTEGER, INTENT(IN) :: nb_procs, bloc_size, m_max_pad
    REAL(KIND=8), DIMENSION(:), OPTIONAL, INTENT(INOUT) :: temps
    REAL(C_DOUBLE), DIMENSION(3), TARGET :: t3
    INTEGER(C_INT) :: rc
    IF (distributed(communicator, nb_procs, 'FFT_PAR_CROSS_PROD_DCL')) THEN
       IF (SIZE(V1_in,2) /= 6 .OR. SIZE(V2_in,2) /= 6) &
            CALL usage_stop('FFT_PAR_CROSS_PROD_DCL', 'the number of slots SIZE(V,2) does not fit the product')
       CALL mode_distributed(communicator, 0, V1_in, 6, V2_in, 6, V_out, 6, 1, SIZE(V1_in,1), SIZE(V1_in,3), &
            nb_procs, bloc_size, m_max_pad, 'FFT_PAR_CROSS_PROD_DCL', temps)
       RETURN
    END IF
    rc = sfnl_fft_par_cross_prod_dcl(V1_in, V2_in, V_out, INT(SIZE(V1_in,1), C_INT), INT(SIZE(V1_in,2), C_INT), &
         INT(SIZE(V1_in,3), C_INT), INT(nb_procs, C_INT), INT(bloc_size, C_INT), INT(m_max_pad, C_INT), C_LOC(t3))
    CALL stop_on_error(rc, 'FFT_PAR_CROSS_PROD_DCL')
    IF (PRESENT(temps)) THEN
       temps = 0.d0
       temps(1:MIN(3,SIZE(temps))) = t3(1:MIN(3,SIZE(temps)))
    END IF
  END SUBROUTINE FFT_PAR_CROSS_PROD_DCL

  SUBROUTINE FFT_PAR_DOT_PROD_DCL(communicator, V1_in, V2_in, c_out, nb_procs, bloc_size, m_max_pad, temps)
    MPI_Comm :: communicator
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V1_in, V2_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: c_out
    INTEGER, INTENT(IN) :: nb_procs, bloc_size, m_max_pad
    REAL(KIND=8), DIMENSION(:), OPTIONAL, INTENT(INOUT) :: temps
    REAL(C_DOUBLE), DIMENSION(3), TARGET :: t3
    INTEGER(C_INT) :: rc
    IF (distributed(communicator, nb_procs, 'FFT_PAR_DOT_PROD_DCL')) THEN
       IF (SIZE(V1_in,2) /= 6 .OR. SIZE(V2_in,2) /= 6) &
            CALL usage_stop('FFT_PAR_DOT_PROD_DCL', 'the number of slots SIZE(V,2) does not fit the product')
       CALL mode_distributed(communicator, 1, V1_in, 6, V2_in, 6, c_out, 2, 1, SIZE(V1_in,1), SIZE(V1_in,3), &
            nb_procs, bloc_size, m_max_pad, 'FFT_PAR_DOT_PROD_DCL', temps)
       RETURN
    END IF
    rc = sfnl_fft_par_dot_prod_dcl(V1_in, V2_in, c_out, INT(SIZE(V1_in,1), C_INT), INT(SIZE(V1_in,2), C_INT), &
         INT(SIZE(V1_in,3), C_INT), INT(nb_procs, C_INT), INT(bloc_size, C_INT), INT(m_max_pad, C_INT), C_LOC(t3))
    CALL stop_on_error(rc, 'FFT_PAR_DOT_PROD_DCL')
    IF (PRESENT(temps)) THEN
       temps = 0.d0
       temps(1:MIN(3,SIZE(temps))) = t3(1:MIN(3,SIZE(temps)))
    END IF
  END SUBROUTINE FFT_PAR_DOT_PROD_DCL

  SUBROUTINE FFT_PAR_PROD_DCL(communicator, c1_in, c2_in, c_out, nb_procs, bloc_size, m_max_pad, temps)
    MPI_Comm :: communicator
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: c1_in, c2_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: c_out
    INTEGER, INTENT(IN) :: nb_procs, bloc_size, m_max_pad
    REAL(KIND=8), DIMENSION(:), OPTIONAL, INTENT(INOUT) :: temps
    REAL(C_DOUBLE), DIMENSION(3), TARGET :: t3
    INTEGER(C_INT) :: rc
    IF (distributed(communicator, nb_procs, 'FFT_PAR_PROD_DCL')) THEN
       IF (SIZE(c1_in,2) /= 2 .OR. SIZE(c2_in,2) /= 2) &
            CALL usage_stop('FFT_PAR_PROD_DCL', 'the number of slots SIZE(V,2) does not fit the product')
       CALL mode_distributed(communicator, 2, c1_in, 2, c2_in, 2, c_out, 2, 1, SIZE(c1_in,1), SIZE(c1_in,3), &
            nb_procs, bloc_size, m_max_pad, 'FFT_PAR_PROD_DCL', temps)
       RETURN
    END IF
    rc = sfnl_fft_par_prod_dcl(c1_in, c2_in, c_out, INT(SIZE(c1_in,1), C_INT), INT(SIZE(c1_in,3), C_INT), &
         INT(nb_procs, C_INT), INT(bloc_size, C_INT), INT(m_max_pad, C_INT), C_LOC(t3))
    CALL stop_on_error(rc, 'FFT_PAR_PROD_DCL')
    IF (PRESENT(temps)) THEN
       temps = 0.d0
       temps(1:MIN(3,SIZE(temps))) = t3(1:MIN(3,SIZE(temps)))
    END IF
  END SUBROUTINE FFT_PAR_PROD_DCL

  SUBROUTINE FFT_PAR_DIV_DCL(communicator, c1_in, c2_in, c_out, nb_procs, bloc_size, m_max_pad, temps)
    MPI_Comm :: communicator
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: c1_in, c2_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: c_out
    INTEGER, INTENT(IN) :: nb_procs, bloc_size, m_max_pad
    REAL(KIND=8), DIMENSION(:), OPTIONAL, INTENT(INOUT) :: temps
    REAL(C_DOUBLE), DIMENSION(3), TARGET :: t3
    INTEGER(C_INT) :: rc
    IF (distributed(communicator, nb_procs, 'FFT_PAR_DIV_DCL')) THEN
       IF (SIZE(c1_in,2) /= 2 .OR. SIZE(c2_in,2) /= 2) &
            CALL usage_stop('FFT_PAR_DIV_DCL', 'the number of slots SIZE(V,2) does not fit the product')
       CALL mode_distributed(communicator, 3, c1_in, 2, c2_in, 2, c_out, 2, 1, SIZE(c1_in,1), SIZE(c1_in,3), &
            nb_procs, bloc_size, m_max_pad, 'FFT_PAR_DIV_DCL', temps)
       RETURN
    END IF
    rc = sfnl_fft_par_div_dcl(c1_in, c2_in, c_out, INT(SIZE(c1_in,1), C_INT), INT(SIZE(c1_in,3), C_INT), &
         INT(nb_procs, C_INT), INT(bloc_size, C_INT), INT(m_max_pad, C_INT), C_LOC(t3))
    CALL stop_on_error(rc, 'FFT_PAR_DIV_DCL')
    IF (PRESENT(temps)) THEN
       temps = 0.d0
       temps(1:MIN(3,SIZE(temps))) = t3(1:MIN(3,SIZE(temps)))
    END IF
  END SUBROUTINE FFT_PAR_DIV_DCL

  SUBROUTINE FFT_SCALAR_VECT_DCL(communicator, V1_in, V2_in, V_out, pb, nb_procs, bloc_size, m_max_pad, temps)
    MPI_Comm :: communicator
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V1_in ! VECTOR
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V2_in ! SCALAR
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: V_out
    INTEGER, INTENT(IN) :: pb, nb_procs, bloc_size, m_max_pad
    REAL(KIND=8), DIMENSION(:), OPTIONAL, INTENT(INOUT) :: temps
    REAL(C_DOUBLE), DIMENSION(3), TARGET :: t3
    INTEGER(C_INT) :: rc
    IF (distributed(communicator, nb_procs, 'FFT_SCALAR_VECT_DCL')) THEN
       IF (SIZE(V1_in,2) /= 6 .OR. SIZE(V2_in,2) /= 2) &
            CALL usage_stop('FFT_SCALAR_VECT_DCL', 'the number of slots SIZE(V,2) does not fit the product')
       IF (pb /= 1 .AND. pb /= 2) CALL usage_stop('FFT_SCALAR_VECT_DCL', 'error in problem type')
       CALL mode_distributed(communicator, 3 + pb, V1_in, 6, V2_in, 2, V_out, 6, 1, SIZE(V1_in,1), SIZE(V1_in,3), &
            nb_procs, bloc_size, m_max_pad, 'FFT_SCALAR_VECT_DCL', temps)
       RETURN
    END IF
    rc = sfnl_fft_scalar_vect_dcl(V1_in, V2_in, V_out, INT(pb, C_INT), INT(SIZE(V1_in,1), C_INT), &
         INT(SIZE(V1_in,2), C_INT), INT(SIZE(V2_in,2), C_INT), INT(SIZE(V1_in,3), C_INT), INT(nb_procs, C_INT), &
         INT(bloc_size, C_INT), INT(m_max_pad, C_INT), C_LOC(t3))
    CALL stop_on_error(rc, 'FFT_SCALAR_VECT_DCL')
    IF (PRESENT(temps)) THEN
       temps = 0.d0
       temps(1:MIN(3,SIZE(temps))) = t3(1:MIN(3,SIZE(temps)))
    END IF
  END SUBROUTINE FFT_SCALAR_VECT_DCL

  SUBROUTINE FFT_TENSOR_DCL(communicator, V1_in, V2_in, V_out, nb_procs, bloc_size, m_max_pad, temps, opt_tension)
    MPI_Comm :: communicator
    REAL(KIND=8), DIMENSION(:,:,:),   CONTIGUOUS, INTENT(IN)  :: V1_in, V2_in
    REAL(KIND=8), DIMENSION(:,:,:,:), CONTIGUOUS, INTENT(OUT) :: V_out
    INTEGER, INTENT(IN) :: nb_procs, bloc_size, m_max_pad
    REAL(KIND=8), DIMENSION(:), OPTIONAL, INTENT(INOUT) :: temps
    LOGICAL,                    OPTIONAL, INTENT(IN)    :: opt_tension
    REAL(C_DOUBLE), DIMENSION(3), TARGET :: t3
    INTEGER(C_INT) :: rc, tension
    tension = -1                     ! absent: plain tensor product
    IF (PRESENT(opt_tension)) THEN
       tension = 0                   ! present and .FALSE.: rejected by the library, as by the reference
       IF (opt_tension) tension = 1
    END IF
    IF (distributed(communicator, nb_procs, 'FFT_TENSOR_DCL')) THEN
       IF (SIZE(V1_in,2) /= 6 .OR. SIZE(V2_in,2) /= 6) &
            CALL usage_stop('FFT_TENSOR_DCL', 'the number of slots SIZE(V,2) does not fit the product')
       IF (tension == 0) CALL usage_stop('FFT_TENSOR_DCL', 'opt_tension should be true if used')
       CALL mode_distributed(communicator, MERGE(7, 6, tension > 0), V1_in, 6, V2_in, 6, V_out, 6, 3, &
            SIZE(V1_in,1), SIZE(V1_in,3), nb_procs, bloc_size, m_max_pad, 'FFT_TENSOR_DCL', temps)
       RETURN
    END IF
    rc = sfnl_fft_tensor_dcl(V1_in, V2_in, V_out, INT(SIZE(V1_in,1), C_INT), INT(SIZE(V1_in,2), C_INT), &
         INT(SIZE(V1_in,3), C_INT), INT(nb_procs, C_INT), INT(bloc_size, C_INT), INT(m_max_pad, C_INT), tension, &
         C_LOC(t3))
    CALL stop_on_error(rc, 'FFT_TENSOR_DCL')
    IF (PRESENT(temps)) THEN
       temps = 0.d0
       temps(1:MIN(3,SIZE(temps))) = t3(1:MIN(3,SIZE(temps)))
    END IF
  END SUBROUTINE FFT_TENSOR_DCL

  SUBROUTINE FFT_PAR_REAL(communicator, V1_in, V_out, opt_nb_plane)
    MPI_Comm :: communicator
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN) :: V1_in
    REAL(KIND=8), DIMENSION(:,:,:), ALLOCATABLE            :: V_out
    INTEGER, OPTIONAL                                      :: opt_nb_plane
    INTEGER(C_INT) :: rc, nplane, n_r
    CALL check_comm(communicator, 1, 'FFT_PAR_REAL')
    nplane = 0
    IF (PRESENT(opt_nb_plane)) nplane = INT(opt_nb_plane, C_INT)
    n_r = sfnl_fft_par_real_planes(INT(SIZE(V1_in,3), C_INT), nplane)
    IF (n_r < 1) CALL stop_on_error(n_r, 'FFT_PAR_REAL')
    IF (ALLOCATED(V_out)) DEALLOCATE(V_out)
    ALLOCATE(V_out(n_r, SIZE(V1_in,2)/2, SIZE(V1_in,1)))
    rc = sfnl_fft_par_real(V1_in, V_out, INT(SIZE(V1_in,1), C_INT), INT(SIZE(V1_in,2), C_INT), &
         INT(SIZE(V1_in,3), C_INT), 1_C_INT, nplane)
    CALL stop_on_error(rc, 'FFT_PAR_REAL')
  END SUBROUTINE FFT_PAR_REAL

  SUBROUTINE FFT_MAX_VEL_DCL(communicator, V1_in, V_out, nb_procs, bloc_size, m_max_pad)
    MPI_Comm :: communicator
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN) :: V1_in
    REAL(KIND=8), INTENT(OUT)                              :: V_out
    INTEGER, INTENT(IN) :: bloc_size, m_max_pad, nb_procs
    REAL(C_DOUBLE) :: vmax
    INTEGER(C_INT) :: rc
    CALL check_comm(communicator, nb_procs, 'FFT_MAX_VEL_DCL')
    rc = sfnl_fft_max_vel_dcl(V1_in, vmax, INT(SIZE(V1_in,1), C_INT), INT(SIZE(V1_in,2), C_INT), &
         INT(SIZE(V1_in,3), C_INT), INT(nb_procs, C_INT), INT(bloc_size, C_INT), INT(m_max_pad, C_INT))
    CALL stop_on_error(rc, 'FFT_MAX_VEL_DCL')
    V_out = vmax
  END SUBROUTINE FFT_MAX_VEL_DCL

END MODULE fft_parallele_gpu

!
! smb_cross_prod_gauss_sft_par_gpu -- the Navier-Stokes caller of the cross product
! (SOURCES/SIMULATION/subroutine_ns_with_velocity.F90:512-629) on the GPU: same arguments as
! smb_cross_prod_gauss_sft_par; the Gauss-point velocity, curl and precession rotation are built
! on the GPU from the nodal V_in and the mesh arrays, then (RotV + 2 Om) x W.  A caller switches by
! calling this routine instead (one Fourier rank).
!
MODULE sfemans_gauss_gpu
#include "petsc/finclude/petsc.h"
  USE petsc
  USE ISO_C_BINDING
  USE def_type_mesh
  USE input_data
  IMPLICIT NONE
  PRIVATE
  PUBLIC :: smb_cross_prod_gauss_sft_par_gpu, smb_CurlH_cross_B_gauss_sft_par_gpu, smb_ugradc_gauss_fft_par_gpu, &
       smb_ugradc_gauss_fft_par_temperature_gpu, smb_ugradc_gauss_fft_par_conc_gpu

  INTERFACE
     FUNCTION sfnl_smb_cross_prod_gauss(V_in, jj, ww, dw, rr, k_d, list_mode, omega, V_out, np_nodes, me, n_w, &
          l_G, nmod, nb_procs) RESULT(rc) BIND(C, NAME='sfnl_smb_cross_prod_gauss')
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: V_in, ww, dw, rr
       INTEGER(C_INT), DIMENSION(*), INTENT(IN)  :: jj, list_mode
       TYPE(C_PTR), VALUE                        :: omega
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: V_out
       INTEGER(C_INT), VALUE :: k_d, np_nodes, me, n_w, l_G, nmod, nb_procs
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_smb_cross_prod_gauss
     FUNCTION sfnl_smb_curlh_cross_b_gauss(V_in, W_in, jj, ww, dw, rr, k_d, list_mode, V_out, np_nodes, me, n_w, &
          l_G, nmod, nb_procs) RESULT(rc) BIND(C, NAME='sfnl_smb_curlh_cross_b_gauss')
       IMPORT :: C_INT, C_DOUBLE
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: V_in, W_in, ww, dw, rr
       INTEGER(C_INT), DIMENSION(*), INTENT(IN)  :: jj, list_mode
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: V_out
       INTEGER(C_INT), VALUE :: k_d, np_nodes, me, n_w, l_G, nmod, nb_procs
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_smb_curlh_cross_b_gauss
     FUNCTION sfnl_smb_ugradc_gauss(V_in, c_in, heat_capa, conservative, jj, ww, dw, rr, k_d, list_mode, c_out, &
          np_nodes, me, n_w, l_G, nmod, nb_procs) RESULT(rc) BIND(C, NAME='sfnl_smb_ugradc_gauss')
       IMPORT :: C_INT, C_DOUBLE, C_PTR
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: V_in, c_in, ww, dw, rr
       TYPE(C_PTR), VALUE                        :: heat_capa
       INTEGER(C_INT), DIMENSION(*), INTENT(IN)  :: jj, list_mode
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: c_out
       INTEGER(C_INT), VALUE :: conservative, k_d, np_nodes, me, n_w, l_G, nmod, nb_procs
       INTEGER(C_INT)        :: rc
     END FUNCTION sfnl_smb_ugradc_gauss
  END INTERFACE

CONTAINS

  SUBROUTINE smb_cross_prod_gauss_sft_par_gpu(communicator, mesh, list_mode, V_in, V_out, precession_in)
    TYPE(mesh_type),                            INTENT(IN)  :: mesh
    INTEGER,      DIMENSION(:),                 INTENT(IN)  :: list_mode
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: V_out
    LOGICAL,                                    INTENT(IN)  :: precession_in
    MPI_Comm :: communicator
    REAL(C_DOUBLE), DIMENSION(:,:,:), ALLOCATABLE, TARGET :: omega
    INTEGER(C_INT), DIMENSION(SIZE(list_mode)) :: modes
    INTEGER(C_INT) :: rc
    INTEGER :: nproc, code, i
    REAL(KIND=8) :: PI
    TYPE(C_PTR) :: om_ptr
    CALL MPI_COMM_SIZE(communicator, nproc, code)
    modes = INT(list_mode, C_INT)
    om_ptr = C_NULL_PTR
    IF (precession_in) THEN  ! the nodal rotation of :540-554
       PI = ACOS(-1.d0)
       ALLOCATE(omega(mesh%np, 6, SIZE(list_mode)))
       omega = 0.d0
       DO i = 1, SIZE(list_mode)
          IF (list_mode(i) == 1) THEN
             omega(:,1,i) = inputs%taux_precession * SIN(inputs%angle_s_pi*PI)
             omega(:,4,i) = -inputs%taux_precession * SIN(inputs%angle_s_pi*PI)
          ELSE IF (list_mode(i) == 0) THEN
             omega(:,5,i) = inputs%taux_precession * COS(inputs%angle_s_pi*PI)
          END IF
       END DO
       om_ptr = C_LOC(omega)
    END IF
    rc = sfnl_smb_cross_prod_gauss(V_in, INT(mesh%jj, C_INT), mesh%gauss%ww, mesh%gauss%dw, mesh%rr, &
         INT(SIZE(mesh%rr,1), C_INT), modes, om_ptr, V_out, INT(mesh%np, C_INT), INT(mesh%me, C_INT), &
         INT(mesh%gauss%n_w, C_INT), INT(mesh%gauss%l_G, C_INT), INT(SIZE(list_mode), C_INT), INT(nproc, C_INT))
    IF (rc /= 0) THEN
       WRITE(*,*) ' BUG in smb_cross_prod_gauss_sft_par_gpu (status ', rc, ')'
       STOP
    END IF
    IF (ALLOCATED(omega)) DEALLOCATE(omega)
  END SUBROUTINE smb_cross_prod_gauss_sft_par_gpu

  ! The Lorentz force (curl H) x B of subroutine_ns_with_m.F90:788-883 (V_in = H, W_in = B).
  SUBROUTINE smb_CurlH_cross_B_gauss_sft_par_gpu(communicator, mesh, list_mode, V_in, W_in, V_out)
    TYPE(mesh_type),                            INTENT(IN)  :: mesh
    INTEGER,      DIMENSION(:),                 INTENT(IN)  :: list_mode
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V_in, W_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS              :: V_out
    MPI_Comm :: communicator
    INTEGER(C_INT) :: rc
    INTEGER :: nproc, code
    CALL MPI_COMM_SIZE(communicator, nproc, code)
    rc = sfnl_smb_curlh_cross_b_gauss(V_in, W_in, INT(mesh%jj, C_INT), mesh%gauss%ww, mesh%gauss%dw, mesh%rr, &
         INT(SIZE(mesh%rr,1), C_INT), INT(list_mode, C_INT), V_out, INT(mesh%np, C_INT), INT(mesh%me, C_INT), &
         INT(mesh%gauss%n_w, C_INT), INT(mesh%gauss%l_G, C_INT), INT(SIZE(list_mode), C_INT), INT(nproc, C_INT))
    IF (rc /= 0) THEN
       WRITE(*,*) ' BUG in smb_CurlH_cross_B_gauss_sft_par_gpu (status ', rc, ')'
       STOP
    END IF
  END SUBROUTINE smb_CurlH_cross_B_gauss_sft_par_gpu

  ! The three advection callers share one entry: heat_capa (C_NULL_PTR: none) and the conservative term.
  ! All mesh%me elements are evaluated (the reference loops over mesh%dom_me, equal to me on these meshes).
  SUBROUTINE ugradc_gpu(mesh, list_mode, V_in, c_in, c_out, heat_ptr, conservative, nproc, who)
    TYPE(mesh_type),                            INTENT(IN)  :: mesh
    INTEGER,      DIMENSION(:),                 INTENT(IN)  :: list_mode
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V_in, c_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: c_out
    TYPE(C_PTR),  INTENT(IN) :: heat_ptr
    INTEGER,      INTENT(IN) :: conservative, nproc
    CHARACTER(*), INTENT(IN) :: who
    INTEGER(C_INT) :: rc
    rc = sfnl_smb_ugradc_gauss(V_in, c_in, heat_ptr, INT(conservative, C_INT), INT(mesh%jj, C_INT), mesh%gauss%ww, &
         mesh%gauss%dw, mesh%rr, INT(SIZE(mesh%rr,1), C_INT), INT(list_mode, C_INT), c_out, INT(mesh%np, C_INT), &
         INT(mesh%me, C_INT), INT(mesh%gauss%n_w, C_INT), INT(mesh%gauss%l_G, C_INT), INT(SIZE(list_mode), C_INT), &
         INT(nproc, C_INT))
    IF (rc /= 0) THEN
       WRITE(*,*) ' BUG in ', who, ' (status ', rc, ')'
       STOP
    END IF
  END SUBROUTINE ugradc_gpu

  ! Level set, subroutine_level_set.F90:434-534: grad c . u.
  SUBROUTINE smb_ugradc_gauss_fft_par_gpu(communicator, mesh, list_mode, V_in, c_in, nb_procs, c_out)
    TYPE(mesh_type),                            INTENT(IN)  :: mesh
    INTEGER,                                    INTENT(IN)  :: nb_procs
    INTEGER,      DIMENSION(:),                 INTENT(IN)  :: list_mode
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V_in, c_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: c_out
    MPI_Comm :: communicator
    CALL ugradc_gpu(mesh, list_mode, V_in, c_in, c_out, C_NULL_PTR, 0, nb_procs, 'smb_ugradc_gauss_fft_par_gpu')
  END SUBROUTINE smb_ugradc_gauss_fft_par_gpu

  ! Temperature, subroutine_temperature_with_T.F90:247-350: (C grad T) . u + div u (C T).
  SUBROUTINE smb_ugradc_gauss_fft_par_temperature_gpu(communicator, mesh, list_mode, heat_capa_in, V_in, c_in, c_out)
    TYPE(mesh_type),                            INTENT(IN)  :: mesh
    INTEGER,      DIMENSION(:),                 INTENT(IN)  :: list_mode
    REAL(KIND=8), DIMENSION(:),     CONTIGUOUS, INTENT(IN), TARGET :: heat_capa_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V_in, c_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: c_out
    MPI_Comm :: communicator
    INTEGER :: nproc, code
    IF (SIZE(heat_capa_in) < mesh%me) THEN
       WRITE(*,*) ' BUG in smb_ugradc_gauss_fft_par_temperature_gpu: heat_capa_in shorter than mesh%me'
       STOP
    END IF
    CALL MPI_COMM_SIZE(communicator, nproc, code)
    CALL ugradc_gpu(mesh, list_mode, V_in, c_in, c_out, C_LOC(heat_capa_in), 1, nproc, &
         'smb_ugradc_gauss_fft_par_temperature_gpu')
  END SUBROUTINE smb_ugradc_gauss_fft_par_temperature_gpu

  ! Concentration, subroutine_concentration.F90:243-341: grad c . u + div u c.
  SUBROUTINE smb_ugradc_gauss_fft_par_conc_gpu(communicator, mesh, list_mode, V_in, c_in, c_out)
    TYPE(mesh_type),                            INTENT(IN)  :: mesh
    INTEGER,      DIMENSION(:),                 INTENT(IN)  :: list_mode
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(IN)  :: V_in, c_in
    REAL(KIND=8), DIMENSION(:,:,:), CONTIGUOUS, INTENT(OUT) :: c_out
    MPI_Comm :: communicator
    INTEGER :: nproc, code
    CALL MPI_COMM_SIZE(communicator, nproc, code)
    CALL ugradc_gpu(mesh, list_mode, V_in, c_in, c_out, C_NULL_PTR, 1, nproc, 'smb_ugradc_gauss_fft_par_conc_gpu')
  END SUBROUTINE smb_ugradc_gauss_fft_par_conc_gpu

END MODULE sfemans_gauss_gpu
