! calexp2t_xm.f90 -- SUBROUTINE CALEXP2T on the GPU: replaces EFDC/calexp2t.f90
! (called at EFDC/hdmt2t.f90:494) for single-layer models (KC = 1) with the
! standard momentum fluxes (IS2LMC = 0) and none of vegetation (ISVEG),
! wave forcing (ISWAVE 2, 4), body forces (ISBODYF), atmospheric pressure
! gradients (IATMP), MHK devices, or momentum of withdrawals and sources
! (NQWRMFU, NQWRMFD, NQSMF): the library computes FCAX, FCAY, FX, FY, CAC and
! FCAXE, FCAYE, FXE, FYE (calexp2t.f90:129-956) and returns them to MODULE
! GLOBAL; the next CALPUV2C call then passes its sums as unchanged, so they
! are not sent back.  With KC > 1 the internal-mode parts of CALEXP2T (the
! vertical fluxes FWU, FWV, the buoyancy forcing and the shears DU, DV) stay
! in the original routine, which such models keep.
! The context is the one of MODULE EFDC_XM_HOST (created here when this runs
! before the first CALPUV2C, as hdmt2t.f90:494-509 orders them).
SUBROUTINE CALEXP2T
  USE GLOBAL
  USE EFDC_XM_BIND
  USE EFDC_XM_HOST
  IMPLICIT NONE

  TYPE(EFDC_XM_MOMENTUM_T) :: MO
  TYPE(EFDC_XM_EXPLICIT_PARAMS_T) :: PRM
  TYPE(EFDC_XM_EXPLICIT_FIELDS_T) :: FLD
  LOGICAL, SAVE :: FIRST = .TRUE.
  INTEGER(C_INT32_T), SAVE, ALLOCATABLE, TARGET :: LHDMFI(:), WETI(:)
  INTEGER :: L, NWR, LL

  IF( KC /= 1 .OR. IS2LMC == 1 .OR. ISVEG > 0 .OR. ISWAVE == 2 .OR. ISWAVE == 4 .OR. &
      ISBODYF > 0 .OR. IATMP > 0 .OR. LMHK )THEN
    STOP '*** CALEXP2T (GPU): needs KC=1, IS2LMC=0, ISVEG=0, ISWAVE<2, ISBODYF=0, IATMP=0, no MHK'
  ENDIF
  DO NWR=1,NQWR
    IF( NQWRMFU(NWR) /= 0 .OR. NQWRMFD(NWR) /= 0 ) &
      STOP '*** CALEXP2T (GPU): withdrawal/return momentum fluxes are not supported'
  ENDDO
  DO LL=1,NQSIJ
    IF( NQSMF(LL) /= 0 ) STOP '*** CALEXP2T (GPU): source momentum fluxes are not supported'
  ENDDO
  CALL XM_OPEN('CALEXP2T')
  IF( FIRST )THEN
    ! *** the static part, once
    ALLOCATE(LHDMFI(LCM), WETI(LCM))
    DO L=1,LCM
      LHDMFI(L) = 0
      IF( LHDMF(L,KC) ) LHDMFI(L) = 1
    ENDDO
    MO%KC = KC
    MO%LD = LCM
    MO%FCORC = C_LOC(FCORC(1));  MO%DYDI = C_LOC(DYDI(1));  MO%DXDJ = C_LOC(DXDJ(1))
    MO%SCAX = C_LOC(SCAX(1));    MO%SCAY = C_LOC(SCAY(1))
    MO%SAAX = C_LOC(SAAX(1));    MO%SAAY = C_LOC(SAAY(1))
    MO%SGZU = C_LOC(SGZU(1,1));  MO%SGZV = C_LOC(SGZV(1,1))
    MO%FSGZU = C_LOC(FSGZU(1,1)); MO%FSGZV = C_LOC(FSGZV(1,1))
    MO%STCUV = C_NULL_PTR
    IF( ITRICELL > 0 ) MO%STCUV = C_LOC(STCUV(1))
    MO%SDX = C_LOC(SDX(1));      MO%SDY = C_LOC(SDY(1))
    MO%LHDMF = C_LOC(LHDMFI(1))
    MO%LNWC = C_LOC(LNWC(1));    MO%LSEC = C_LOC(LSEC(1))
    MO%NBCS = NBCS
    MO%PAD_ = 0
    MO%LBCS = C_LOC(LBCS(1));    MO%LBERC = C_LOC(LBERC(1));  MO%LBNRC = C_LOC(LBNRC(1))
    IF( EFDC_XM_SET_MOMENTUM(XM_CTX, 0_C_INT32_T, MO) /= EFDC_XM_OK )THEN
      WRITE(6,'(2A)') ' CALEXP2T (GPU): ', TRIM(EFDC_XM_ERRMSG())
      STOP '*** CALEXP2T (GPU): static part not accepted'
    ENDIF
    FIRST = .FALSE.
  ENDIF

  PRM%SNLT = SNLT
  PRM%ISCURVATURE = 0
  IF( ISCURVATURE ) PRM%ISCURVATURE = 1
  PRM%ISHDMF = ISHDMF

  FLD%U = C_LOC(U(1,1));       FLD%V = C_LOC(V(1,1))
  FLD%UHDY = C_LOC(UHDY(1,1)); FLD%VHDX = C_LOC(VHDX(1,1))
  FLD%HP = C_LOC(HP(1))
  ! *** the wet set LWET of the last CALPUV2C (all cells without wetting and drying)
  FLD%WET = C_NULL_PTR
  IF( ISDRY > 0 )THEN
    DO L=1,LCM
      WETI(L) = 0
      IF( LMASKDRY(L) ) WETI(L) = 1
    ENDDO
    FLD%WET = C_LOC(WETI(1))
  ENDIF
  FLD%FUHJ = C_NULL_PTR;  FLD%FVHJ = C_NULL_PTR
  FLD%FMDUX = C_NULL_PTR; FLD%FMDUY = C_NULL_PTR
  FLD%FMDVX = C_NULL_PTR; FLD%FMDVY = C_NULL_PTR
  IF( ISHDMF >= 1 )THEN
    FLD%FMDUX = C_LOC(FMDUX(1,1)); FLD%FMDUY = C_LOC(FMDUY(1,1))
    FLD%FMDVX = C_LOC(FMDVX(1,1)); FLD%FMDVY = C_LOC(FMDVY(1,1))
  ENDIF
  FLD%FCAXE = C_LOC(FCAXE(1)); FLD%FCAYE = C_LOC(FCAYE(1))
  FLD%FXE = C_LOC(FXE(1));     FLD%FYE = C_LOC(FYE(1))
  FLD%FCAX = C_LOC(FCAX(1,1)); FLD%FCAY = C_LOC(FCAY(1,1))
  FLD%FX = C_LOC(FX(1,1));     FLD%FY = C_LOC(FY(1,1))
  FLD%CAC = C_LOC(CAC(1,1))
  IF( EFDC_XM_EXPLICIT(XM_CTX, PRM, FLD) /= EFDC_XM_OK )THEN
    WRITE(6,'(2A)') ' CALEXP2T (GPU): ', TRIM(EFDC_XM_ERRMSG())
    STOP '*** CALEXP2T (GPU) FAILED'
  ENDIF
  ! *** the sums in MODULE GLOBAL are the device's: the next step need not send them
  XM_SUMS_ON_DEVICE = .TRUE.
END SUBROUTINE CALEXP2T
