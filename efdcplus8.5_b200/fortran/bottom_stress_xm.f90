! bottom_stress_xm.f90 -- the bottom stresses on the GPU: replaces, at
! EFDC/hdmt2t.f90:669-684, CALL CALTBXY(ISTL,IS2TL) and the TBX/TBY loop after
! it by CALL BOTTOM_STRESS_XM(ISTL,IS2TL), for models whose drag is CALTBXY's
! bed form alone (ISWAVE=0, ISVEG=0, ISMUD=0, ISITB=0, MDCHH=0) on the standard
! sigma grid.  The library computes STBX, STBY (caltbxy.f90:476-539) and TBX,
! TBY (hdmt2t.f90:670-684) from the state its last step left on the device and
! keeps TBX, TBY there; the host copies come back for the internal mode.
! The context is the one of MODULE EFDC_XM_HOST (CALPUV2C or CALPUV9C).
SUBROUTINE BOTTOM_STRESS_XM(ISTL_, IS2TL_)
  USE GLOBAL
  USE EFDC_XM_BIND
  USE EFDC_XM_HOST
  IMPLICIT NONE

  INTEGER, INTENT(IN) :: ISTL_, IS2TL_
  TYPE(EFDC_XM_BED_T) :: BED
  TYPE(EFDC_XM_DRAG_PARAMS_T) :: PRM
  TYPE(EFDC_XM_DRAG_FIELDS_T) :: FLD
  LOGICAL, SAVE :: FIRST = .TRUE.
  REAL(C_DOUBLE), SAVE, ALLOCATABLE, TARGET :: STBXO_(:), STBYO_(:)
  INTEGER :: L

  IF( ISWAVE > 0 .OR. ISVEG > 0 .OR. ISMUD > 0 .OR. ISITB > 0 .OR. MDCHH > 0 &
      .OR. .NOT. C_ASSOCIATED(XM_CTX) )THEN
    STOP '*** BOTTOM_STRESS_XM: needs ISWAVE=ISVEG=ISMUD=ISITB=0, MDCHH=0 and a first step'
  ENDIF
  IF( FIRST )THEN
    ! *** the bed, once: STBX, STBY as read are the multipliers (caltbxy.f90:108-116)
    ALLOCATE(STBXO_(LCM), STBYO_(LCM))
    DO L=1,LCM
      STBXO_(L) = STBX(L)
      STBYO_(L) = STBY(L)
    ENDDO
    BED%ZBR = C_LOC(ZBR(1))
    BED%STBXO = C_LOC(STBXO_(1));  BED%STBYO = C_LOC(STBYO_(1))
    BED%DXP = C_LOC(DXP(1));       BED%DYP = C_LOC(DYP(1))
    BED%DZC1 = C_LOC(DZC(1,1))
    BED%SGZU1 = C_LOC(SGZU(1,1));  BED%SGZV1 = C_LOC(SGZV(1,1))
    BED%KC = KC
    BED%PAD_ = 0
    BED%AVCON = AVCON
    BED%VISMUD = VISMUD
    BED%COEFTSBL = COEFTSBL
    IF( EFDC_XM_SET_BED(XM_CTX, 0_C_INT32_T, BED) /= EFDC_XM_OK )THEN
      WRITE(6,'(2A)') ' BOTTOM_STRESS_XM: ', TRIM(EFDC_XM_ERRMSG())
      STOP '*** BOTTOM_STRESS_XM: bed not accepted'
    ENDIF
    FIRST = .FALSE.
  ENDIF

  ! *** DELT of CALTBXY (caltbxy.f90:56-66)
  PRM%DELT = DT2
  IF( ISTL_ /= 3 ) PRM%DELT = DT
  IF( IS2TL_ == 1 )THEN
    IF( ISDYNSTP == 0 )THEN
      PRM%DELT = DT
    ELSE
      PRM%DELT = DTDYN
    ENDIF
  ENDIF
  PRM%AVCON1 = AVCON1
  PRM%ISDRY = ISDRY
  PRM%N = N
  PRM%NTSTBC = NTSTBC
  PRM%PAD_ = 0

  ! *** layer 1 is the bottom layer on the standard sigma grid (KSZU = KSZV = 1)
  FLD%UB = C_LOC(U(1,1));   FLD%VB = C_LOC(V(1,1))
  FLD%VU = C_LOC(VU(1));    FLD%UV = C_LOC(UV(1))
  FLD%H1U = C_LOC(H1U(1));  FLD%H1V = C_LOC(H1V(1))
  FLD%STBX = C_LOC(STBX(1)); FLD%STBY = C_LOC(STBY(1))
  FLD%TBX = C_LOC(TBX(1));   FLD%TBY = C_LOC(TBY(1))
  IF( EFDC_XM_BOTTOM_STRESS(XM_CTX, PRM, FLD) /= EFDC_XM_OK )THEN
    WRITE(6,'(2A)') ' BOTTOM_STRESS_XM: ', TRIM(EFDC_XM_ERRMSG())
    STOP '*** BOTTOM_STRESS_XM FAILED'
  ENDIF
END SUBROUTINE BOTTOM_STRESS_XM
