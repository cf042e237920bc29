! efdc_xm_host.f90 -- the host side shared by the drop-ins of CALPUV2C
! (calpuv2c_xm.f90) and CALPUV9C (calpuv9c_xm.f90):
!   * XM_OPEN: the library context, created once from MODULE GLOBAL (replaces
!     the first-call blocks, calpuv2c.f90:59-126 and calpuv9c.f90:38-103), with
!     the sigma layers (BSC > 1E-6) and the sub-grid channels (MDCHH >= 1);
!   * XM_FIELDS: the per-call scalars and arrays both steps pass;
!   * XM_FINISH: LOGICAL arrays back, the reference's STOP / EFDCLOG.OUT /
!     EE_LINKAGE behaviour on failure (congrad.f90:171-184,
!     calpuv2c.f90:726-749, calpuv9c.f90:770-790), the wet lists LKWET/LLWET,
!     SUB3D/SVB3D (calpuv2c.f90:958-1187), the layer depths of the cells whose
!     volume was wasted (calpuv2c.f90:874-878, 1010-1015), and the
!     negative-depth message of NEGDEP.
! The implicit bottom and vegetation drag (ISITB>=1, ISVEG>0) pass their
! inputs: the bottom-layer velocities U(L,KSZU(L)), V(L,KSZV(L)) gathered per
! cell, VU, UV, STBX, STBY, FXVEGE, FYVEGE (calpuv2c.f90:222-243).
! Restrictions (the library returns EFDC_XM_UNSUPPORTED or XM_OPEN stops):
! ISGWIE=0, IGRIDV=0 (the baroclinic terms of BSC>1E-6 on
! the standard sigma grid), no periodic (ISCONNECT) links; sub-grid channels
! (MDCHH>=1) of MDCHTYP 1 and 2, whose cells are not open-boundary cells.
MODULE EFDC_XM_HOST
  USE GLOBAL
  USE EFDCOUT
  USE EFDC_XM_BIND
  IMPLICIT NONE

  TYPE(C_PTR), SAVE :: XM_CTX = C_NULL_PTR
  TYPE(EFDC_XM_GRID_T), SAVE, TARGET :: XM_GRD
  REAL(C_DOUBLE), SAVE, ALLOCATABLE, TARGET :: PSERW(:), PSERE(:), PSERS(:), PSERN(:)
  INTEGER(C_INT32_T), SAVE, ALLOCATABLE, TARGET :: LMASKI(:), ISCDRYI(:), LOBCDRYI(:)
  REAL(C_DOUBLE), SAVE, ALLOCATABLE, TARGET :: UBOTI(:), VBOTI(:)
  ! set by the CALEXP2T drop-in: FCAXE, FCAYE, FXE, FYE hold what the library
  ! computed and returned, so the next step passes them as unchanged
  LOGICAL, SAVE :: XM_SUMS_ON_DEVICE = .FALSE.

CONTAINS

  SUBROUTINE XM_OPEN(WHO)
    CHARACTER(*), INTENT(IN) :: WHO
    TYPE(EFDC_XM_CHANNELS_T) :: CHN
    TYPE(EFDC_XM_LAYERS_T) :: LYR

    IF( ISGWIE > 0 .OR. IGRIDV > 0 )THEN
      WRITE(6,'(2A)') WHO, ' (GPU): ISGWIE, IGRIDV options are not supported'
      STOP '*** EXTERNAL MODE (GPU): unsupported options'
    ENDIF
    IF( C_ASSOCIATED(XM_CTX) ) RETURN

    XM_GRD%LA = LA
    XM_GRD%LC = LC
    XM_GRD%IL = C_LOC(IL(1));     XM_GRD%JL = C_LOC(JL(1))
    XM_GRD%LNC = C_LOC(LNC(1));   XM_GRD%LSC = C_LOC(LSC(1))
    XM_GRD%LEC = C_LOC(LEC(1));   XM_GRD%LWC = C_LOC(LWC(1))
    XM_GRD%DXYP = C_LOC(DXYP(1)); XM_GRD%DXYIP = C_LOC(DXYIP(1))
    XM_GRD%DXIU = C_LOC(DXIU(1)); XM_GRD%DYIU = C_LOC(DYIU(1))
    XM_GRD%DXIV = C_LOC(DXIV(1)); XM_GRD%DYIV = C_LOC(DYIV(1))
    XM_GRD%DXYU = C_LOC(DXYU(1)); XM_GRD%DXYV = C_LOC(DXYV(1))
    XM_GRD%HRUO = C_LOC(HRUO(1)); XM_GRD%HRVO = C_LOC(HRVO(1))
    XM_GRD%SUBO = C_LOC(SUBO(1)); XM_GRD%SVBO = C_LOC(SVBO(1))
    XM_GRD%SBXO = C_LOC(SBXO(1)); XM_GRD%SBYO = C_LOC(SBYO(1))
    XM_GRD%BELV = C_LOC(BELV(1))
    XM_GRD%MTIDE = MTIDE
    XM_GRD%TCP = C_LOC(TCP(1))
    XM_GRD%OBC(1) = EFDC_XM_OBC_T(NPBW, C_LOC(LPBW(1)), C_LOC(ISPBW(1)), C_LOC(PCBW(1,1)), C_LOC(PSBW(1,1)), SIZE(PCBW,1))
    XM_GRD%OBC(2) = EFDC_XM_OBC_T(NPBE, C_LOC(LPBE(1)), C_LOC(ISPBE(1)), C_LOC(PCBE(1,1)), C_LOC(PSBE(1,1)), SIZE(PCBE,1))
    XM_GRD%OBC(3) = EFDC_XM_OBC_T(NPBS, C_LOC(LPBS(1)), C_LOC(ISPBS(1)), C_LOC(PCBS(1,1)), C_LOC(PSBS(1,1)), SIZE(PCBS,1))
    XM_GRD%OBC(4) = EFDC_XM_OBC_T(NPBN, C_LOC(LPBN(1)), C_LOC(ISPBN(1)), C_LOC(PCBN(1,1)), C_LOC(PSBN(1,1)), SIZE(PCBN,1))
    XM_CTX = EFDC_XM_CREATE(XM_GRD, 0_C_INT32_T)
    IF( .NOT. C_ASSOCIATED(XM_CTX) )THEN
      WRITE(6,'(3A)') WHO, ' (GPU): ', TRIM(EFDC_XM_ERRMSG())
      STOP '*** EXTERNAL MODE (GPU): context creation failed'
    ENDIF
    IF( BSC > 1.E-6 )THEN
      ! *** layers of the sigma grid for CALEBI (aaefdc.f90:1090-1237)
      LYR%KC = KC
      LYR%LD = LCM
      LYR%DZC = C_LOC(DZC(1,1))
      LYR%ZZ = C_LOC(ZZ(1,1))
      IF( EFDC_XM_SET_LAYERS(XM_CTX, 0_C_INT32_T, LYR) /= EFDC_XM_OK )THEN
        WRITE(6,'(3A)') WHO, ' (GPU): ', TRIM(EFDC_XM_ERRMSG())
        STOP '*** EXTERNAL MODE (GPU): layers not accepted'
      ENDIF
    ENDIF
    IF( MDCHH >= 1 )THEN
      ! *** sub-grid channels (input.f90:2563-2590, ainit.f90:286-316)
      CHN%N = MDCHH
      CHN%TYPE = C_LOC(MDCHTYP(1)); CHN%LHOST = C_LOC(LMDCHH(1))
      CHN%LU = C_LOC(LMDCHU(1));    CHN%LV = C_LOC(LMDCHV(1))
      CHN%CHANLEN = C_LOC(CHANLEN(1)); CHN%CHANFRIC = C_LOC(CHANFRIC(1))
      CHN%DXP = C_LOC(DXP(1));      CHN%DYP = C_LOC(DYP(1))
      IF( EFDC_XM_SET_CHANNELS(XM_CTX, 0_C_INT32_T, CHN) /= EFDC_XM_OK )THEN
        WRITE(6,'(3A)') WHO, ' (GPU): ', TRIM(EFDC_XM_ERRMSG())
        STOP '*** EXTERNAL MODE (GPU): sub-grid channels not accepted'
      ENDIF
    ENDIF
    ALLOCATE(PSERW(MAX(NPBW,1)), PSERE(MAX(NPBE,1)), PSERS(MAX(NPBS,1)), PSERN(MAX(NPBN,1)))
    ALLOCATE(LMASKI(LCM), ISCDRYI(LCM), LOBCDRYI(LCM))
    ALLOCATE(UBOTI(LCM), VBOTI(LCM))
    UBOTI = 0.0
    VBOTI = 0.0
  END SUBROUTINE XM_OPEN

  ! The scalars and arrays both steps pass; the caller sets DELT, TN and the
  ! three-time-level members afterwards.
  SUBROUTINE XM_FIELDS(PRM, FLD)
    TYPE(EFDC_XM_PARAMS_T), INTENT(OUT) :: PRM
    TYPE(EFDC_XM_FIELDS_T), INTENT(OUT) :: FLD
    INTEGER :: L, LL

    PRM%G = G
    PRM%HDRY = HDRY
    PRM%RSQM = RSQM
    PRM%PI2 = PI2
    PRM%SNLT = SNLT
    PRM%RITB1 = RITB1
    PRM%ITERM = ITERM
    PRM%ISDRY = ISDRY
    PRM%NDRYSTP = NDRYSTP
    PRM%ISBAL = ISBAL
    PRM%N = N
    PRM%NTSTBC = NTSTBC
    PRM%MAX_SWEEPS = 500
    PRM%PRECISION = EFDC_XM_PREC_FP64
    PRM%MIXED_RSQ_FACTOR = 0.0
    PRM%QCHERR = QCHERR
    PRM%CHAN_CONSISTENT = 0     ! CONGRADC as the reference writes it
    PRM%PAD_ = 0
    PRM%BSC = BSC
    PRM%GP = GP
    PRM%TL3_ISTL = 0
    PRM%NCTBC = 0
    PRM%ROLD = 0.0
    PRM%RNEW = 1.0
    PRM%ISITB = ISITB
    PRM%ISVEG = ISVEG
    PRM%RITB = RITB

    ! *** time series part of the open-boundary targets (setopenbc.f90:41-46)
    DO LL=1,NPBW
      PSERW(LL) = PSERT(NPSERW(LL)) + 0.5*PSERZDF(NPSERW(LL)) + PSERST(NPSERW(LL)) + 0.5*PSERZDS(NPSERW(LL))
    ENDDO
    DO LL=1,NPBE
      PSERE(LL) = PSERT(NPSERE(LL)) + 0.5*PSERZDF(NPSERE(LL)) + PSERST(NPSERE(LL)) + 0.5*PSERZDS(NPSERE(LL))
    ENDDO
    DO LL=1,NPBS
      PSERS(LL) = PSERT(NPSERS(LL)) + 0.5*PSERZDF(NPSERS(LL)) + PSERST(NPSERS(LL)) + 0.5*PSERZDS(NPSERS(LL))
    ENDDO
    DO LL=1,NPBN
      PSERN(LL) = PSERT(NPSERN(LL)) + 0.5*PSERZDF(NPSERN(LL)) + PSERST(NPSERN(LL)) + 0.5*PSERZDS(NPSERN(LL))
    ENDDO

    ! *** LOGICAL arrays travel as 0/1 integers; OLDMASK is the mask at entry
    ! *** (calpuv2c.f90:178)
    DO L=1,LC
      IF( ISDRY > 0 ) OLDMASK(L) = LMASKDRY(L)
      LMASKI(L) = MERGE(1, 0, LMASKDRY(L))
      LOBCDRYI(L) = MERGE(1, 0, LOPENBCDRY(L))
      ISCDRYI(L) = ISCDRY(L)
    ENDDO

    FLD%P = C_LOC(P(1));         FLD%HP = C_LOC(HP(1));       FLD%H1P = C_LOC(H1P(1))
    FLD%HU = C_LOC(HU(1));       FLD%HV = C_LOC(HV(1))
    FLD%UHDYE = C_LOC(UHDYE(1)); FLD%VHDXE = C_LOC(VHDXE(1))
    FLD%SUB = C_LOC(SUB(1));     FLD%SVB = C_LOC(SVB(1))
    FLD%SBX = C_LOC(SBX(1));     FLD%SBY = C_LOC(SBY(1))
    FLD%LMASKDRY = C_LOC(LMASKI(1));  FLD%ISCDRY = C_LOC(ISCDRYI(1))
    FLD%LOPENBCDRY = C_LOC(LOBCDRYI(1)); FLD%NATDRY = C_LOC(NATDRY(1))
    FLD%FCAXE = C_LOC(FCAXE(1)); FLD%FCAYE = C_LOC(FCAYE(1))
    FLD%FXE = C_LOC(FXE(1));     FLD%FYE = C_LOC(FYE(1))
    FLD%TSX = C_LOC(TSX(1));     FLD%TSY = C_LOC(TSY(1))
    FLD%TBX = C_LOC(TBX(1));     FLD%TBY = C_LOC(TBY(1))
    FLD%QSUME = C_LOC(QSUME(1))
    FLD%PSER(1) = C_LOC(PSERW(1)); FLD%PSER(2) = C_LOC(PSERE(1))
    FLD%PSER(3) = C_LOC(PSERS(1)); FLD%PSER(4) = C_LOC(PSERN(1))
    FLD%UHE = C_LOC(UHE(1));     FLD%VHE = C_LOC(VHE(1))
    FLD%HPI = C_LOC(HPI(1));     FLD%HUI = C_LOC(HUI(1));     FLD%HVI = C_LOC(HVI(1))
    FLD%QDWASTE = C_LOC(QDWASTE(1)); FLD%VDWASTE = C_LOC(VDWASTE(1))
    FLD%LWET = C_LOC(LWET(1));   FLD%LDRY = C_LOC(LDRY(1))
    FLD%CCC = C_NULL_PTR; FLD%CCS = C_NULL_PTR; FLD%CCW = C_NULL_PTR
    FLD%CCE = C_NULL_PTR; FLD%CCN = C_NULL_PTR; FLD%FPTMP = C_NULL_PTR
    IF( MDCHH >= 1 )THEN
      FLD%QCHANU = C_LOC(QCHANU(1));   FLD%QCHANV = C_LOC(QCHANV(1))
      FLD%QCHANUN = C_LOC(QCHANUN(1)); FLD%QCHANVN = C_LOC(QCHANVN(1))
    ELSE
      FLD%QCHANU = C_NULL_PTR;  FLD%QCHANV = C_NULL_PTR
      FLD%QCHANUN = C_NULL_PTR; FLD%QCHANVN = C_NULL_PTR
    ENDIF
    IF( BSC > 1.E-6 )THEN
      FLD%B = C_LOC(B(1,1))
      FLD%B_LD = LCM
    ELSE
      FLD%B = C_NULL_PTR
      FLD%B_LD = 0
    ENDIF
    FLD%PAD_B_ = 0
    FLD%P1 = C_NULL_PTR;     FLD%H2P = C_NULL_PTR
    FLD%UHDY1E = C_NULL_PTR; FLD%VHDX1E = C_NULL_PTR
    FLD%UHDY2E = C_NULL_PTR; FLD%VHDX2E = C_NULL_PTR
    FLD%H1U = C_NULL_PTR;    FLD%H1V = C_NULL_PTR
    FLD%TSX1 = C_NULL_PTR;   FLD%TSY1 = C_NULL_PTR
    FLD%TBX1 = C_NULL_PTR;   FLD%TBY1 = C_NULL_PTR
    FLD%FPGXE = C_NULL_PTR;  FLD%FPGYE = C_NULL_PTR
    IF( ISITB >= 1 .OR. ISVEG > 0 )THEN
      ! *** the implicit drag's inputs (calpuv2c.f90:222-243): the bottom layer's
      ! *** velocities per cell, the rest as MODULE GLOBAL holds them
      DO L=2,LA
        UBOTI(L) = U(L,KSZU(L))
        VBOTI(L) = V(L,KSZV(L))
      ENDDO
      FLD%UBOT = C_LOC(UBOTI(1)); FLD%VBOT = C_LOC(VBOTI(1))
      FLD%VU = C_LOC(VU(1));      FLD%UV = C_LOC(UV(1))
      FLD%STBX = C_LOC(STBX(1));  FLD%STBY = C_LOC(STBY(1))
      IF( ISVEG > 0 )THEN
        FLD%FXVEGE = C_LOC(FXVEGE(1)); FLD%FYVEGE = C_LOC(FYVEGE(1))
      ELSE
        FLD%FXVEGE = C_NULL_PTR;       FLD%FYVEGE = C_NULL_PTR
      ENDIF
    ELSE
      FLD%UBOT = C_NULL_PTR; FLD%VBOT = C_NULL_PTR; FLD%VU = C_NULL_PTR; FLD%UV = C_NULL_PTR
      FLD%STBX = C_NULL_PTR; FLD%STBY = C_NULL_PTR
      FLD%FXVEGE = C_NULL_PTR; FLD%FYVEGE = C_NULL_PTR
    ENDIF
    FLD%UNCHANGED = 0    ! every array is sent each step, but the sums of the CALEXP2T drop-in
    IF( XM_SUMS_ON_DEVICE ) FLD%UNCHANGED = IOR(IOR(EFDC_XM_SAME_FCAXE, EFDC_XM_SAME_FCAYE), &
                                                IOR(EFDC_XM_SAME_FXE, EFDC_XM_SAME_FYE))
    XM_SUMS_ON_DEVICE = .FALSE.
    FLD%PAD_U_ = 0
  END SUBROUTINE XM_FIELDS

  SUBROUTINE XM_FINISH(IRC, ST, WHO)
    INTEGER(C_INT32_T), INTENT(IN) :: IRC
    TYPE(EFDC_XM_STATS_T), INTENT(IN) :: ST
    CHARACTER(*), INTENT(IN) :: WHO
    INTEGER :: L, K, ND, LF, LP, LN
    REAL :: HWASTE

    DO L=2,LA
      LMASKDRY(L) = LMASKI(L) /= 0
      LOPENBCDRY(L) = LOBCDRYI(L) /= 0
      ISCDRY(L) = ISCDRYI(L)
    ENDDO
    IDRYTBP = ST%ITERS_LAST
    ITER = ST%ITERS_LAST

    SELECT CASE (IRC)
    CASE (EFDC_XM_OK, EFDC_XM_NEG_DEPTH)
      CONTINUE
    CASE (EFDC_XM_CG_MAXITER)                   ! congrad.f90:171-184
      WRITE(6,'(A)') '  MAXIMUM ITERATIONS EXCEEDED IN EXTERNAL SOLUTION'
      OPEN(8,FILE=OUTDIR//'EFDCLOG.OUT',POSITION='APPEND')
      WRITE(8,'(A)') '  MAXIMUM ITERATIONS EXCEEDED IN EXTERNAL SOLUTION (GPU)'
      CLOSE(8)
      CALL EE_LINKAGE(-1)
      STOP
    CASE (EFDC_XM_WETDRY_MAXSWEEP)              ! calpuv2c.f90:726-749
      OPEN(8,FILE=OUTDIR//'EFDCLOG.OUT',POSITION='APPEND')
      IF( ISPPH == 1 ) CALL EE_LINKAGE(-1)
      CLOSE(8)
      STOP '*** NCORDRY > 500 WHEN ISDRY > 0'
    CASE DEFAULT
      WRITE(6,'(2A,I3,2A)') WHO, ' (GPU) ERROR ', IRC, ': ', TRIM(EFDC_XM_ERRMSG())
      STOP '*** EXTERNAL MODE (GPU) FAILED'
    END SELECT

    ! *** wet cell counts and per-layer lists (calpuv2c.f90:1061-1187)
    IF( ISDRY == 0 )THEN
      LAWET = LA-1
      LADRY = 0
    ELSE
      LAWET = ST%LAWET
      LADRY = ST%LADRY
    ENDIF
    LDMWET = INT(FLOAT(LAWET)/FLOAT(NDM))+1
    LDMDRY = INT(FLOAT(LADRY)/FLOAT(NDM))+1
    IF( ISDRY > 0 )THEN
      DO ND=1,NDM
        LF=(ND-1)*LDMWET+1
        DO K=1,KC
          LN=0
          DO LP=LF,MIN(LF+LDMWET-1,LAWET)
            L=LWET(LP)
            IF( LKSZ(L,K) )CYCLE
            LN = LN+1
            LKWET(LN,K,ND)=L
          ENDDO
          LLWET(K,ND)=LN
        ENDDO
      ENDDO
      DO K=1,KC
        DO L=2,LA
          IF( LKSZ(L,K) )CYCLE
          SUB3D(L,K) = SUB(L)*SUB3DO(L,K)
          SVB3D(L,K) = SVB(L)*SVB3DO(L,K)
        ENDDO
      ENDDO
    ENDIF

    ! *** the layer depths of the cells whose volume was wasted: the library
    ! *** leaves HP = H1P = 0.9*HDRY there (calpuv2c.f90:874-878, 1010-1015)
    IF( ST%N_WASTED > 0 )THEN
      HWASTE = 0.90*HDRY
      DO L=2,LA
        IF( HP(L) == HWASTE .AND. H1P(L) == HWASTE )THEN
          DO K=KSZ(L),KC
            HPK(L,K)  = HP(L)*DZC(L,K)
            HPKI(L,K) = 1./HPK(L,K)
            H1PK(L,K) = H1P(L)*DZC(L,K)
          ENDDO
        ENDIF
      ENDDO
    ENDIF

    ! *** negative depths: diagnostics as NEGDEP does (negdep.f90:47-167)
    IF( IRC == EFDC_XM_NEG_DEPTH )THEN
      WRITE(6,'(A,I8,A,F12.4)') ' NEGATIVE DEPTH IN ', ST%N_NEGDEP, ' CELLS AT TIMEDAY ', TIMEDAY
    ENDIF
  END SUBROUTINE XM_FINISH

END MODULE EFDC_XM_HOST
