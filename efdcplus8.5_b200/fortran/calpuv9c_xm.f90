! calpuv9c_xm.f90 -- drop-in replacement of EFDC/calpuv9c.f90 (SUBROUTINE
! CALPUV9C(ISTL_), the external mode of the three-time-level scheme, called at
! EFDC/hdmt.f90:415).
!
! The step runs on the GPU through libefdc_xm (efdc_xm_step with
! tl3_istl = ISTL_): the leapfrog step over DT2 (ISTL_ = 3) with its advance
! of the 2D levels (UHDY2E <- UHDY1E <- UHDYE, P1 <- P, H1U <- HU, H1V <- HV,
! H2P <- H1P <- HP, calpuv9c.f90:282-311), or the trapezoidal correction over
! DT (ISTL_ = 2).  This shim keeps the copies of that advance the library does
! not make (U1V, V1U, H1UI, H1VI and the KC-layer arrays H2PK, H1PK, UHDY2EK,
! VHDX2EK, UHDY1EK, VHDX1EK, calpuv9c.f90:296-318); the rest of the host side
! (context, failure behaviour, wet lists) is MODULE EFDC_XM_HOST.
SUBROUTINE CALPUV9C(ISTL_)
  USE GLOBAL
  USE EFDC_XM_BIND
  USE EFDC_XM_HOST
  IMPLICIT NONE

  INTEGER, INTENT(IN) :: ISTL_
  TYPE(EFDC_XM_PARAMS_T) :: PRM
  TYPE(EFDC_XM_FIELDS_T), TARGET :: FLD
  TYPE(EFDC_XM_STATS_T) :: ST
  INTEGER :: L, K
  INTEGER(C_INT32_T) :: IRC

  CALL XM_OPEN('CALPUV9C')
  CALL XM_FIELDS(PRM, FLD)

  ! *** per-call scalars (calpuv9c.f90:105-111, setopenbc.f90:22-23)
  IF( ISTL_ == 2 )THEN
    PRM%DELT = DT
  ELSE
    PRM%DELT = DT2
  ENDIF
  PRM%TN = DT*FLOAT(N) + TCON*TBEGIN
  PRM%TL3_ISTL = ISTL_
  PRM%NCTBC = NCTBC
  PRM%ROLD = ROLD
  PRM%RNEW = RNEW

  FLD%P1 = C_LOC(P1(1));         FLD%H2P = C_LOC(H2P(1))
  FLD%UHDY1E = C_LOC(UHDY1E(1)); FLD%VHDX1E = C_LOC(VHDX1E(1))
  FLD%UHDY2E = C_LOC(UHDY2E(1)); FLD%VHDX2E = C_LOC(VHDX2E(1))
  FLD%H1U = C_LOC(H1U(1));       FLD%H1V = C_LOC(H1V(1))
  FLD%TSX1 = C_LOC(TSX1(1));     FLD%TSY1 = C_LOC(TSY1(1))
  FLD%TBX1 = C_LOC(TBX1(1));     FLD%TBY1 = C_LOC(TBY1(1))
  IF( BSC > 1.E-6 )THEN
    FLD%FPGXE = C_LOC(FPGXE(1)); FLD%FPGYE = C_LOC(FPGYE(1))
  ENDIF

  IF( ISTL_ == 3 )THEN
    ! *** the copies of the level advance the library does not make
    ! *** (calpuv9c.f90:296-318; HUI, HVI and the layer arrays at entry)
    DO L=2,LA
      U1V(L) = UV(L)
      V1U(L) = VU(L)
      H1UI(L) = HUI(L)
      H1VI(L) = HVI(L)
    ENDDO
    DO K=1,KC
      DO L=2,LA
        H2PK(L,K) = H1PK(L,K)
        H1PK(L,K) = HPK(L,K)
        UHDY2EK(L,K) = UHDY1EK(L,K)
        VHDX2EK(L,K) = VHDX1EK(L,K)
        UHDY1EK(L,K) = UHDYEK(L,K)
        VHDX1EK(L,K) = VHDXEK(L,K)
      ENDDO
    ENDDO
  ENDIF

  IRC = EFDC_XM_STEP(XM_CTX, PRM, FLD, ST)
  CALL XM_FINISH(IRC, ST, 'CALPUV9C')
END SUBROUTINE CALPUV9C
