! calpuv2c_xm.f90 -- drop-in replacement of EFDC/calpuv2c.f90 (SUBROUTINE
! CALPUV2C, no arguments, called at EFDC/hdmt2t.f90:509).
!
! The external-mode step runs on the GPU through libefdc_xm (efdc_xm_step).
! This shim keeps what belongs to the host side of EFDC+: the layer copies of
! the time-level advance (calpuv2c.f90:256-274 for the KC-layer arrays
! H1PK/UHDY1EK/VHDX1EK) and the 2D copies of the levels the library does not
! return (UHDY1E, VHDX1E, P1, H1U, H1V, H1UI, H1VI, H2P); the rest of the host
! side (context, failure behaviour, wet lists) is MODULE EFDC_XM_HOST.
SUBROUTINE CALPUV2C
  USE GLOBAL
  USE EFDC_XM_BIND
  USE EFDC_XM_HOST
  IMPLICIT NONE

  TYPE(EFDC_XM_PARAMS_T) :: PRM
  TYPE(EFDC_XM_FIELDS_T), TARGET :: FLD
  TYPE(EFDC_XM_STATS_T) :: ST
  INTEGER :: L, K
  INTEGER(C_INT32_T) :: IRC

  CALL XM_OPEN('CALPUV2C')
  CALL XM_FIELDS(PRM, FLD)

  ! *** per-call scalars (calpuv2c.f90:128-136, setopenbc.f90:22-23)
  IF( ISDYNSTP == 0 )THEN
    PRM%DELT = DT
    PRM%TN = DT*FLOAT(N) + TCON*TBEGIN
  ELSE
    PRM%DELT = DTDYN
    PRM%TN = TIMESEC
  ENDIF
  DELT = PRM%DELT
  DELTD2 = 0.5*DELT
  DELTI = 1./DELT
  ISTL = 2
  PRM%TL3_ISTL = 0            ! CALPUV2C: two time levels

  ! *** 2D time levels the library does not return (calpuv2c.f90:256-266)
  DO L=2,LA
    UHDY1E(L) = UHDYE(L)
    VHDX1E(L) = VHDXE(L)
    P1(L) = P(L)
    H1U(L) = HU(L)
    H1V(L) = HV(L)
    H1UI(L) = HUI(L)
    H1VI(L) = HVI(L)
    H2P(L) = H1P(L)
  ENDDO
  DO K=1,KC
    DO L=2,LA
      H1PK(L,K) = HPK(L,K)
      UHDY1EK(L,K) = UHDYEK(L,K)
      VHDX1EK(L,K) = VHDXEK(L,K)
    ENDDO
  ENDDO

  IRC = EFDC_XM_STEP(XM_CTX, PRM, FLD, ST)
  CALL XM_FINISH(IRC, ST, 'CALPUV2C')
END SUBROUTINE CALPUV2C
