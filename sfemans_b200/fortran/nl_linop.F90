!
! nl_linop -- the linearised dealiased cross product as a LightKrylov linear operator.
!
! SFEMaNS's stability and adjoint computations drive LightKrylov operators: the reference's
! exptA_linop (SOURCES/LIGHTKRYLOV_OBJECTS/exponential_propagator.F90:53-63) extends
! abstract_exptA_linop_rdp and binds rmatvec to the forward matvec, since the reference has no
! adjoint.  This module provides the building block that operator lacks: the Jacobian of the
! nonlinear term N(u, w) = u x w (FFT_PAR_CROSS_PROD_DCL, fft_parallel.F90:147-328) about a base
! state, with matvec = JVP (du, dw) -> du x w + u x dw and rmatvec = its exact transpose (VJP),
! both evaluated on the GPU by libsfemans_nl.so (sfnl_cross_jvp_host, sfnl_cross_vjp_host).
!
! The operator maps coefficient arrays (np, 12, m) -> (np, 6, m): it is rectangular, so it serves
! LightKrylov's general solvers (svds, lsqr) as an abstract_linop_rdp; the stability operator of
! eigs needs the linearised time stepper around it, which is the caller's.
!
! Written against LightKrylov's abstract_vector_rdp / abstract_linop_rdp interfaces (zero, rand,
! scal, axpby, dot, get_size; matvec, rmatvec), the library the reference builds with
! USE_LIGHTKRYLOV (LIBS/CMakeLists.txt:33-45).  Not compiled here: neither gfortran nor LightKrylov
! is installed on the machines this repository was built and tested on.
!
MODULE nl_linop
#ifdef USE_LIGHTKRYLOV
  USE LightKrylov, ONLY: abstract_vector_rdp, abstract_linop_rdp
#endif
  USE ISO_C_BINDING
  IMPLICIT NONE
  PRIVATE

#ifdef USE_LIGHTKRYLOV
  ! A coefficient array V(np, nslot, m) in the reference's layout, as a LightKrylov vector.
  TYPE, EXTENDS(abstract_vector_rdp), PUBLIC :: coef_vector
     REAL(KIND=8), ALLOCATABLE, DIMENSION(:,:,:) :: v
   CONTAINS
     PROCEDURE, PASS(self), PUBLIC :: zero => cv_zero
     PROCEDURE, PASS(self), PUBLIC :: rand => cv_rand
     PROCEDURE, PASS(self), PUBLIC :: scal => cv_scal
     PROCEDURE, PASS(self), PUBLIC :: axpby => cv_axpby
     PROCEDURE, PASS(self), PUBLIC :: dot => cv_dot
     PROCEDURE, PASS(self), PUBLIC :: get_size => cv_get_size
  END TYPE coef_vector

  ! J(du, dw) = du x w + u x dw about the base state (u, w), each (np, 6, m).
  TYPE, EXTENDS(abstract_linop_rdp), PUBLIC :: cross_jacobian_linop
     REAL(KIND=8), POINTER, DIMENSION(:,:,:) :: u => NULL(), w => NULL()
     INTEGER :: m_max_pad = 0
   CONTAINS
     PROCEDURE, PASS(self), PUBLIC :: matvec => cj_matvec
     PROCEDURE, PASS(self), PUBLIC :: rmatvec => cj_rmatvec
  END TYPE cross_jacobian_linop
#endif

  INTERFACE
     FUNCTION sfnl_cross_jvp_host(u, w, tan, out, np, m_max, m_max_pad, k_batch) RESULT(rc) &
          BIND(C, NAME='sfnl_cross_jvp_host')
       IMPORT :: C_INT, C_INT64_T, C_DOUBLE
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: u, w, tan
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: out
       INTEGER(C_INT64_T), VALUE :: np
       INTEGER(C_INT), VALUE     :: m_max, m_max_pad, k_batch
       INTEGER(C_INT)            :: rc
     END FUNCTION sfnl_cross_jvp_host

     FUNCTION sfnl_cross_vjp_host(u, w, cot, out, np, m_max, m_max_pad, k_batch) RESULT(rc) &
          BIND(C, NAME='sfnl_cross_vjp_host')
       IMPORT :: C_INT, C_INT64_T, C_DOUBLE
       REAL(C_DOUBLE), DIMENSION(*), INTENT(IN)  :: u, w, cot
       REAL(C_DOUBLE), DIMENSION(*), INTENT(OUT) :: out
       INTEGER(C_INT64_T), VALUE :: np
       INTEGER(C_INT), VALUE     :: m_max, m_max_pad, k_batch
       INTEGER(C_INT)            :: rc
     END FUNCTION sfnl_cross_vjp_host
  END INTERFACE

  PUBLIC :: sfnl_cross_jvp_host, sfnl_cross_vjp_host

#ifdef USE_LIGHTKRYLOV
CONTAINS

  SUBROUTINE cv_zero(self)
    CLASS(coef_vector), INTENT(INOUT) :: self
    IF (ALLOCATED(self%v)) self%v = 0.d0
  END SUBROUTINE cv_zero

  SUBROUTINE cv_rand(self, ifnorm)
    CLASS(coef_vector), INTENT(INOUT) :: self
    LOGICAL, OPTIONAL,  INTENT(IN)    :: ifnorm
    REAL(KIND=8) :: nrm
    CALL RANDOM_NUMBER(self%v)
    self%v = self%v - 0.5d0
    self%v(:, 2::2, 1) = 0.d0  ! the sine of mode 0 carries nothing (fft_parallel.F90:241)
    IF (PRESENT(ifnorm)) THEN
       IF (ifnorm) THEN
          nrm = SQRT(SUM(self%v**2))
          IF (nrm > 0.d0) self%v = self%v / nrm
       END IF
    END IF
  END SUBROUTINE cv_rand

  SUBROUTINE cv_scal(self, alpha)
    CLASS(coef_vector), INTENT(INOUT) :: self
    REAL(KIND=8),       INTENT(IN)    :: alpha
    self%v = alpha * self%v
  END SUBROUTINE cv_scal

  ! self = alpha * self + beta * vec
  SUBROUTINE cv_axpby(self, alpha, vec, beta)
    CLASS(coef_vector),         INTENT(INOUT) :: self
    REAL(KIND=8),               INTENT(IN)    :: alpha, beta
    CLASS(abstract_vector_rdp), INTENT(IN)    :: vec
    SELECT TYPE (vec)
    TYPE IS (coef_vector)
       self%v = alpha * self%v + beta * vec%v
    END SELECT
  END SUBROUTINE cv_axpby

  REAL(KIND=8) FUNCTION cv_dot(self, vec) RESULT(d)
    CLASS(coef_vector),         INTENT(IN) :: self
    CLASS(abstract_vector_rdp), INTENT(IN) :: vec
    d = 0.d0
    SELECT TYPE (vec)
    TYPE IS (coef_vector)
       d = SUM(self%v * vec%v)
    END SELECT
  END FUNCTION cv_dot

  INTEGER FUNCTION cv_get_size(self) RESULT(n)
    CLASS(coef_vector), INTENT(IN) :: self
    n = SIZE(self%v)
  END FUNCTION cv_get_size

  SUBROUTINE check(rc, what)
    INTEGER(C_INT),   INTENT(IN) :: rc
    CHARACTER(LEN=*), INTENT(IN) :: what
    IF (rc /= 0) THEN
       WRITE(*,*) ' BUG in ', what, ' (status ', rc, ')'
       STOP
    END IF
  END SUBROUTINE check

  ! vec_in = (du, dw) of shape (np, 12, m); vec_out = du x w + u x dw of shape (np, 6, m)
  SUBROUTINE cj_matvec(self, vec_in, vec_out)
    CLASS(cross_jacobian_linop), INTENT(INOUT) :: self
    CLASS(abstract_vector_rdp),  INTENT(IN)    :: vec_in
    CLASS(abstract_vector_rdp),  INTENT(OUT)   :: vec_out
    INTEGER :: np, m
    np = SIZE(self%u, 1)
    m = SIZE(self%u, 3)
    SELECT TYPE (vec_in)
    TYPE IS (coef_vector)
       SELECT TYPE (vec_out)
       TYPE IS (coef_vector)
          IF (.NOT. ALLOCATED(vec_out%v)) ALLOCATE(vec_out%v(np, 6, m))
          CALL check(sfnl_cross_jvp_host(self%u, self%w, vec_in%v, vec_out%v, INT(np, C_INT64_T), INT(m, C_INT), &
               INT(self%m_max_pad, C_INT), 1_C_INT), 'cross_jacobian_linop%matvec')
       END SELECT
    END SELECT
  END SUBROUTINE cj_matvec

  ! vec_in = c of shape (np, 6, m); vec_out = J^T c of shape (np, 12, m)
  SUBROUTINE cj_rmatvec(self, vec_in, vec_out)
    CLASS(cross_jacobian_linop), INTENT(INOUT) :: self
    CLASS(abstract_vector_rdp),  INTENT(IN)    :: vec_in
    CLASS(abstract_vector_rdp),  INTENT(OUT)   :: vec_out
    INTEGER :: np, m
    np = SIZE(self%u, 1)
    m = SIZE(self%u, 3)
    SELECT TYPE (vec_in)
    TYPE IS (coef_vector)
       SELECT TYPE (vec_out)
       TYPE IS (coef_vector)
          IF (.NOT. ALLOCATED(vec_out%v)) ALLOCATE(vec_out%v(np, 12, m))
          CALL check(sfnl_cross_vjp_host(self%u, self%w, vec_in%v, vec_out%v, INT(np, C_INT64_T), INT(m, C_INT), &
               INT(self%m_max_pad, C_INT), 1_C_INT), 'cross_jacobian_linop%rmatvec')
       END SELECT
    END SELECT
  END SUBROUTINE cj_rmatvec
#endif

END MODULE nl_linop
