/*
 * efdc_xm.h -- C-ABI of the B200 external-mode free-surface solver.
 *
 * Drop-in for EFDC+ 8.5's 2TL external mode:
 *   SUBROUTINE CALPUV2C        EFDC/calpuv2c.f90:1-1191  (called at EFDC/hdmt2t.f90:509)
 *   SUBROUTINE CONGRAD         EFDC/congrad.f90:1-191    (called at EFDC/calpuv2c.f90:409)
 *   SUBROUTINE SETOPENBC(2)    EFDC/setopenbc.f90, EFDC/setopenbc2.f90
 *   SUBROUTINE NEGDEP (check)  EFDC/negdep.f90:34-45
 *
 * Conventions
 *   - Every per-cell array is the base address of the Fortran array indexed
 *     1..LC (or 1..LCM): element L lives at ptr[L-1].  Cells L=2..LA are water
 *     cells in CELLMAP order (EFDC/cellmap.f90:13-28); L=1 and L=LC are the
 *     ghost cells, and a missing neighbour is LC (EFDC/cellmap.f90:80-134).
 *   - Reals are double (the ReleaseDP64 build: /real_size:64).
 *   - Fortran LOGICAL(4) is passed as int32_t: nonzero = .TRUE. on input;
 *     the library writes 1 for .TRUE. and 0 for .FALSE.
 *   - No call aborts the process: failures that STOP in the reference are
 *     returned as a status code (enum efdc_xm_status) and the last message is
 *     available from efdc_xm_last_error().
 *   - A context is bound to one CUDA device and is not thread-safe; use one
 *     context per host thread.  Calls return after the device work finished.
 *
 * The library has no PyTorch dependency.
 */
#ifndef EFDC_XM_H
#define EFDC_XM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EFDC_XM_ABI_VERSION 7

/* Status codes.  The reference STOPs where these are returned. */
enum efdc_xm_status {
  EFDC_XM_OK = 0,
  EFDC_XM_CG_MAXITER = 1,      /* RSQ > RSQM after ITERM iterations: congrad.f90:171-184 */
  EFDC_XM_WETDRY_MAXSWEEP = 2, /* NCORDRY reached 500: calpuv2c.f90:597-601, 726-749      */
  EFDC_XM_NEG_DEPTH = 3,       /* some HP <= 0 after the step: negdep.f90:34-45 (non-fatal) */
  EFDC_XM_NONFINITE = 4,       /* NaN/Inf in the CG scalars or in the new P                  */
  EFDC_XM_CUDA_ERROR = 5,
  EFDC_XM_DEVICE_TIMEOUT = 6,  /* a bounded device-side wait ran out                          */
  EFDC_XM_BAD_ARGUMENT = 7,
  EFDC_XM_UNSUPPORTED = 8      /* an option this library does not implement (see message)    */
};

/* Arithmetic of the solve. */
enum efdc_xm_precision {
  EFDC_XM_PREC_FP64 = 0,  /* FP64 assembly and FP64 Jacobi-PCG, as the DP build          */
  EFDC_XM_PREC_MIXED = 1  /* FP64 assembly; FP32 inner PCG with FP64 dot products inside
                             FP64 iterative refinement r = b - A P; P stays FP64          */
};

/* One side of open (elevation) boundary cells, e.g. NPBW/LPBW/ISPBW/PCBW/PSBW. */
typedef struct efdc_xm_obc {
  int32_t n;           /* NPBW: number of cells on this side                           */
  const int32_t *l;    /* LPBW(1..n): L index of each boundary cell (setbcs.f90:178)  */
  const int32_t *ispb; /* ISPBW(1..n): 0 clamped, 1/2 radiation (setopenbc.f90:54)   */
  const double *pcb;   /* PCBW(LL,M): cosine amplitude G*A*cos(phase), column-major   */
  const double *psb;   /* PSBW(LL,M): sine amplitude   G*A*sin(phase)                 */
  int32_t ld;          /* leading dimension of pcb/psb (NPBWM); >= n                   */
} efdc_xm_obc;

enum { EFDC_XM_OBC_W = 0, EFDC_XM_OBC_E = 1, EFDC_XM_OBC_S = 2, EFDC_XM_OBC_N = 3 };

/* Static model description: copied by efdc_xm_create, not referenced afterwards. */
typedef struct efdc_xm_grid {
  int32_t la;                          /* LA: last water cell                        */
  int32_t lc;                          /* LC = LA+1: ghost cell                      */
  const int32_t *il, *jl;              /* IL, JL (cellmap.f90:18-19)                 */
  const int32_t *lnc, *lsc, *lec, *lwc;/* neighbour maps (cellmap.f90:80-134)        */
  const double *dxyp, *dxyip;          /* aaefdc.f90:2171-2190 metrics               */
  const double *dxiu, *dyiu, *dxiv, *dyiv, *dxyu, *dxyv;
  const double *hruo, *hrvo;           /* HRUO=SUBO*DYU/DXU, HRVO=SVBO*DXV/DYV       */
  const double *subo, *svbo, *sbxo, *sbyo; /* permanent face switches (setbcs.f90:1052) */
  const double *belv;                  /* bed elevation                              */
  int32_t mtide;                       /* number of harmonic constituents            */
  const double *tcp;                   /* TCP(1..mtide): periods (s)                 */
  efdc_xm_obc obc[4];                  /* W, E, S, N open boundaries                 */
} efdc_xm_grid;

/* Per-call scalars (values of MODULE GLOBAL at the call). */
typedef struct efdc_xm_params {
  double delt;       /* DELT: DT, or DTDYN when ISDYNSTP/=0 (calpuv2c.f90:128-136)   */
  double g;          /* G                                                             */
  double hdry;       /* HDRY                                                          */
  double rsqm;       /* RSQM: absolute squared-residual stop of CONGRAD               */
  double tn;         /* TN of SETOPENBC: DT*N+TCON*TBEGIN, or TIMESEC                 */
  double pi2;        /* PI2 = 2*PI with PI=3.1415926535898 (aaefdc.f90:650-651)       */
  double snlt;       /* SNLT                                                          */
  double ritb1;      /* RITB1 (1.0 when ISITB=0, caltbxy.f90:104)                     */
  int32_t iterm;     /* ITERM: CG iteration cap                                       */
  int32_t isdry;     /* ISDRY: 0, 1..97 (legacy) or 99                                */
  int32_t ndrystp;   /* NDRYSTP (<0: waste volume of isolated cells)                  */
  int32_t isbal;     /* ISBAL (keeps QDWASTE when > 0)                                */
  int32_t n;         /* N, time step counter (for the LDRY list rule)                 */
  int32_t ntstbc;    /* NTSTBC                                                        */
  int32_t max_sweeps;/* wet/dry re-solve cap; the reference uses 500                  */
  int32_t precision; /* enum efdc_xm_precision (ignored by the CPU oracle)             */
  double mixed_rsq_factor; /* MIXED only: stop when the FP64 RSQ <= factor*RSQM; 0 selects
                              the default 0.1 (the FP32 path converges a little past
                              RSQM so that its per-step surface error against the FP64
                              solve stays well inside 1e-6 m)                         */
  double qcherr;     /* QCHERR: implicit weight RLAMN of the sub-grid channel flows
                        (calpuv2c.f90:353-354); used only where channels are set      */
  int32_t chan_consistent; /* channels only.  0: CONGRADC as written, which adds the
                        coupling CCCCHH with the same sign to the initial residual
                        (congradc.f90:59-77) and to A*p (:99-116), so that its CG
                        solves (A+C)P = b + 2C*P0 rather than (A-C)P = b (P0: P at
                        entry); the flows it gives can grow without bound.  1: the
                        conductance operator (A-C)P = b, i.e. A*p with -CCCCHH     */
  int32_t pad_;
  double bsc;        /* BSC: the baroclinic terms FPGXE, FPGYE enter when > 1e-6
                        (calpuv2c.f90:161, 192-211); needs efdc_xm_set_layers and B */
  double gp;         /* GP (hdmt2t.f90:459-463)                                       */
  int32_t tl3_istl;  /* 0: CALPUV2C, the two-time-level step (hdmt2t.f90:509).  3 or 2:
                        CALPUV9C(ISTL_) of the three-time-level scheme (hdmt.f90:415):
                        3 the leapfrog step, 2 its trapezoidal correction.  delt is then
                        the DELT of that call (calpuv9c.f90:105-111: DT2 = 2*DT for 3,
                        DT for 2), and the fields' three-time-level arrays are used.
                        All members of a batch take the same value                    */
  int32_t nctbc;     /* NCTBC (CALPUV9C, ISTL_ = 3): 1 halves UHDYE, VHDXE before they
                        become UHDY1E, VHDX1E (calpuv9c.f90:289-294)                   */
  double rold, rnew; /* ROLD, RNEW (CALPUV9C, BSC > 1e-6): FPGXE = ROLD*FPGXE +
                        RNEW*(new gradient) (calpuv9c.f90:157-163; hdmt.f90:304-305,
                        1018-1028: 0 and 1 for ISTL_ = 3, 0.5 and 0.5 for 2)          */
  int32_t isitb;     /* ISITB >= 1: implicit bottom drag with vegetation, RCX, RCY of
                        calpuv2c.f90:222-233 (calpuv9c.f90:220-231); RITB1 is then
                        caltbxy.f90:95-100's (0.45 or 0) and TBX, TBY the explicit part */
  int32_t isveg;     /* ISVEG > 0 (with ISITB = 0): implicit vegetation drag only,
                        calpuv2c.f90:234-242                                         */
  double ritb;       /* RITB (caltbxy.f90:95-105): weight of the implicit bottom drag */
} efdc_xm_params;

/* Per-call arrays.  "in/out" arrays are read and overwritten.  Optional outputs
 * may be NULL. */
typedef struct efdc_xm_fields {
  /* state, in/out */
  double *p, *hp, *h1p;               /* P, HP, H1P (H1P <- HP at entry, calpuv2c.f90:264) */
  double *hu, *hv;                    /* HU, HV (recomputed at exit, :896-899)       */
  double *uhdye, *vhdxe;              /* UHDYE, VHDXE face discharges                */
  double *sub, *svb, *sbx, *sby;      /* face switches (wet/dry changes them)        */
  int32_t *lmaskdry;                  /* LMASKDRY (LOGICAL)                          */
  int32_t *iscdry;                    /* ISCDRY                                      */
  int32_t *lopenbcdry;                /* LOPENBCDRY (LOGICAL)                        */
  int32_t *natdry;                    /* NATDRY (isolated-step counter)              */
  /* explicit terms from the upstream producers, in */
  const double *fcaxe, *fcaye, *fxe, *fye;
  const double *tsx, *tsy, *tbx, *tby;
  const double *qsume;
  /* per open-boundary cell: PSERT+0.5*PSERZDF+PSERST+0.5*PSERZDS (with the
   * NPFORT coordinate blend already applied), i.e. FP(L) before the harmonic
   * sum of setopenbc.f90:47-52.  NULL = zero. */
  const double *pser[4];
  /* outputs */
  double *uhe, *vhe;                  /* unit-width discharges (:432-435)            */
  double *hpi, *hui, *hvi;            /* reciprocals (:902-906)                      */
  double *qdwaste, *vdwaste;          /* volume wasting (NDRYSTP<0), optional        */
  int32_t *lwet, *ldry;               /* LWET(1..LAWET), LDRY(1..LADRY), optional    */
  /* optional diagnostics: the scaled system of the last sweep, as CONGRAD saw it */
  double *ccc, *ccs, *ccw, *cce, *ccn, *fptmp;
  /* sub-grid channels (efdc_xm_set_channels), one element per channel NMD,
   * in/out: QCHANU, QCHANV (the flows of the previous step in, the new ones
   * out, calpuv2c.f90:440-460) and QCHANUN, QCHANVN (set to zero where a
   * channel is inactive, else left as they are).  Required where channels
   * are set, ignored elsewhere. */
  double *qchanu, *qchanv, *qchanun, *qchanvn;
  /* buoyancy B(L,K), in, K = 1..KC of efdc_xm_set_layers, at b[(K-1)*b_ld + L-1]
   * (a Fortran B(LCM,KCM) has b_ld = LCM).  Required where BSC > 1e-6. */
  const double *b;
  int32_t b_ld;
  int32_t pad_b_;
  /* three time levels (tl3_istl = 2 or 3), required there and ignored by CALPUV2C
   * steps.  in/out: ISTL_ = 3 advances them (calpuv9c.f90:288-311: UHDY2E <-
   * UHDY1E <- UHDYE, P1 <- P, H1U <- HU, H1V <- HV, H2P <- H1P <- HP); H1P is then
   * an input as well.  The layer copies (H1PK, UHDY1EK, ...), U1V, V1U, H1UI and
   * H1VI stay with the caller. */
  double *p1, *h2p;                   /* P1, H2P                                      */
  double *uhdy1e, *vhdx1e;            /* UHDY1E, VHDX1E                               */
  double *uhdy2e, *vhdx2e;            /* UHDY2E, VHDX2E                               */
  double *h1u, *h1v;                  /* H1U, H1V                                     */
  const double *tsx1, *tsy1, *tbx1, *tby1;  /* TSX1, TSY1, TBX1, TBY1, in            */
  double *fpgxe, *fpgye;              /* FPGXE, FPGYE, in/out; required where BSC > 1e-6 */
  /* implicit drag (params.isitb >= 1 or params.isveg > 0), in: U(L,KSZU(L)) and
   * V(L,KSZV(L)), the bottom-layer velocities; VU, UV; STBX, STBY (the bed drag
   * coefficients of CALTBXY); FXVEGE, FYVEGE (the vegetative resistance, NULL =
   * 0).  UHE, VHE above are then also read at entry (calpuv2c.f90:226-227).
   * The drag coefficients RCX, RCY stay on the device between steps, as the
   * reference's module arrays do. */
  const double *ubot, *vbot, *vu, *uv, *stbx, *stby, *fxvege, *fyvege;
  /* in, optional (0: every given array is sent): bits of enum efdc_xm_same.
   * A set bit promises that the caller's array holds exactly what this
   * context last uploaded from it or downloaded into it; the library then
   * skips its upload if its own device copy is still that transfer's (no step
   * has written it since without a download).  No counterpart in the
   * reference: it spares a host whose other modules did not touch an array
   * between two steps the copy of it.  The members of a batch give the same
   * bits. */
  uint32_t unchanged;
  int32_t pad_u_;
} efdc_xm_fields;

/* Bits of efdc_xm_fields.unchanged, one per array. */
enum efdc_xm_same {
  EFDC_XM_SAME_P = 1 << 0, EFDC_XM_SAME_HP = 1 << 1, EFDC_XM_SAME_HU = 1 << 2,
  EFDC_XM_SAME_HV = 1 << 3, EFDC_XM_SAME_UHDYE = 1 << 4, EFDC_XM_SAME_VHDXE = 1 << 5,
  EFDC_XM_SAME_SUB = 1 << 6, EFDC_XM_SAME_SVB = 1 << 7, EFDC_XM_SAME_SBX = 1 << 8,
  EFDC_XM_SAME_SBY = 1 << 9, EFDC_XM_SAME_LMASKDRY = 1 << 10, EFDC_XM_SAME_ISCDRY = 1 << 11,
  EFDC_XM_SAME_LOPENBCDRY = 1 << 12, EFDC_XM_SAME_NATDRY = 1 << 13,
  EFDC_XM_SAME_FCAXE = 1 << 14, EFDC_XM_SAME_FCAYE = 1 << 15, EFDC_XM_SAME_FXE = 1 << 16,
  EFDC_XM_SAME_FYE = 1 << 17, EFDC_XM_SAME_TSX = 1 << 18, EFDC_XM_SAME_TSY = 1 << 19,
  EFDC_XM_SAME_TBX = 1 << 20, EFDC_XM_SAME_TBY = 1 << 21, EFDC_XM_SAME_QSUME = 1 << 22,
  EFDC_XM_SAME_QDWASTE = 1 << 23, EFDC_XM_SAME_VDWASTE = 1 << 24
};

typedef struct efdc_xm_stats {
  int32_t status;       /* enum efdc_xm_status                                   */
  int32_t iters_last;   /* IDRYTBP: CG iterations of the last solve              */
  int32_t iters_total;  /* CG iterations summed over the wet/dry sweeps          */
  int32_t solves;       /* CONGRAD calls (1 + NCORDRY)                           */
  int32_t lawet, ladry; /* LAWET, LADRY                                          */
  int32_t n_negdep;     /* cells with HP <= 0                                    */
  int32_t n_wasted;     /* cells whose volume was wasted (NNATDRY)               */
  int32_t outer_refinements; /* MIXED: FP64 refinement passes                    */
  double rsq_last;      /* RSQ at exit of the last solve                         */
  double ccmnm_last;    /* CCMNM of the last sweep                               */
} efdc_xm_stats;

typedef struct efdc_xm_ctx efdc_xm_ctx;

/* Sub-grid channels: MDCHH host-guest pairs whose exchange flow enters the
 * external solve implicitly (subchan.f90:1-124; calpuv2c.f90:139-145,
 * 352-356, 401-410, 440-460, 538-556) and the operator CONGRADC solves
 * (congradc.f90:1-207).  Arrays of n elements, channel NMD at [NMD-1]. */
typedef struct efdc_xm_channels {
  int32_t n;               /* MDCHH (0: no channels)                                  */
  const int32_t *type;     /* MDCHTYP: 1 x-direction (guest LMDCHU), 2 y-direction
                              (guest LMDCHV); other types are not supported          */
  const int32_t *lhost;    /* LMDCHH                                                  */
  const int32_t *lu, *lv;  /* LMDCHU, LMDCHV (1 where unused, as input.f90 sets them) */
  const double *chanlen;   /* CHANLEN as ainit.f90:286-316 leaves it                 */
  const double *chanfric;  /* CHANFRIC                                                */
  const double *dxp, *dyp; /* DXP, DYP of the model (1-based, LC elements): the
                              guest cells' widths and lengths                         */
} efdc_xm_channels;

/* Version of this header the library was built with. */
int32_t efdc_xm_abi_version(void);

/* Last error message of the calling thread ("" if none). */
const char *efdc_xm_last_error(void);

/* Create a solver context on CUDA device `device` for the static model `grid`.
 * Replaces the first-call block of CALPUV2C (calpuv2c.f90:59-126) and the
 * static arrays of MODULE GLOBAL it reads.  Returns NULL on failure. */
efdc_xm_ctx *efdc_xm_create(const efdc_xm_grid *grid, int32_t device);

void efdc_xm_destroy(efdc_xm_ctx *ctx);

/* One external-mode step on host arrays: CALL CALPUV2C (hdmt2t.f90:509).
 * Uploads the fields, runs the whole step on the GPU (assembly, open BCs,
 * scaling, PCG, back-substitution, continuity, wet/dry sweeps, finalisation,
 * wet lists, negative-depth check) and writes the outputs back. */
int32_t efdc_xm_step(efdc_xm_ctx *ctx, const efdc_xm_params *prm,
                     efdc_xm_fields *f, efdc_xm_stats *stats);

/* Device-resident form of efdc_xm_step for callers that keep the state on the
 * GPU between steps: upload once, step many times, download when needed. */
int32_t efdc_xm_upload(efdc_xm_ctx *ctx, const efdc_xm_fields *f);
int32_t efdc_xm_step_device(efdc_xm_ctx *ctx, const efdc_xm_params *prm,
                            efdc_xm_stats *stats);
int32_t efdc_xm_download(efdc_xm_ctx *ctx, efdc_xm_fields *f);

/* Sets (n > 0) or removes (n == 0) the sub-grid channels of member `member`
 * of the context (0 for a single-basin context): the input of
 * calpuv2c.f90:139-145 and subchan.f90.  The host and guest cells must be
 * water cells (2..LA) that are not open-boundary cells, and differ.  A step
 * of a member with channels solves CONGRADC's system in place of CONGRAD's
 * (calpuv2c.f90:409-410) and needs the QCHANU..QCHANVN fields. */
int32_t efdc_xm_set_channels(efdc_xm_ctx *ctx, int32_t member, const efdc_xm_channels *ch);

/* Layer geometry of the standard sigma grid (IGRIDV = 0, KSZ = 1) for the
 * external buoyancy integrals of CALEBI (calebi.f90:82-120): DZC(L,K) and
 * ZZ(L,K), K = 1..kc, at [(K-1)*ld + L-1] (ld = LCM for Fortran arrays;
 * ZZ from its layer 1, i.e. C_LOC(ZZ(1,1))).  kc is shared by the members
 * of a batch (1..64). */
typedef struct efdc_xm_layers {
  int32_t kc;
  int32_t ld;
  const double *dzc, *zz;
} efdc_xm_layers;
int32_t efdc_xm_set_layers(efdc_xm_ctx *ctx, int32_t member, const efdc_xm_layers *ly);

/* Bottom stress producer: CALTBXY's bed drag coefficients STBX, STBY
 * (caltbxy.f90:455-537 for ISWAVE = 0, ISVEG = 0, ISMUD = 0, ISITB = 0: the
 * rough log-law form where ZBR > 1e-6, the smooth viscous form elsewhere)
 * and the bottom stresses TBX, TBY of hdmt2t.f90:670-684, computed on the
 * device from the state the last step left there (HU, HV, LMASKDRY and the
 * entry mask) and the bottom-layer velocities of the internal mode.  The
 * stresses stay on the device for the next step: a step given TBX, TBY = NULL
 * then uses them without an upload.  No reference counterpart as a separate
 * call: it replaces CALL CALTBXY(ISTL,IS2TL) and the TBX/TBY loop at
 * hdmt2t.f90:669-684 when the external mode runs on the GPU. */
typedef struct efdc_xm_bed {        /* static, per member (efdc_xm_set_bed)        */
  const double *zbr;                /* ZBR(L), bed roughness height                */
  const double *stbxo, *stbyo;      /* STBX, STBY as read (the multipliers STBXO,
                                       STBYO of caltbxy.f90:84-87)                 */
  const double *dxp, *dyp;          /* DXP, DYP                                    */
  const double *dzc1;               /* DZC(L,1): thickness fraction of layer 1     */
  const double *sgzu1, *sgzv1;      /* SGZU(L,1), SGZV(L,1) (caltbxy.f90:71-76)    */
  int32_t kc;                       /* KC (1: the single-layer form, :518-526)     */
  int32_t pad_;
  double avcon;                     /* AVCON                                       */
  double vismud, coeftsbl;          /* VISMUD, COEFTSBL (the smooth form)          */
} efdc_xm_bed;
int32_t efdc_xm_set_bed(efdc_xm_ctx *ctx, int32_t member, const efdc_xm_bed *bed);

typedef struct efdc_xm_drag_params { /* per member and call                       */
  double delt;                      /* DELT of CALTBXY (caltbxy.f90:30-42)        */
  double avcon1;                    /* AVCON1 (hdmt2t.f90:682)                     */
  int32_t isdry, n, ntstbc, pad_;   /* ISDRY, N, NTSTBC: the dry-cell list LDRY   */
} efdc_xm_drag_params;

typedef struct efdc_xm_drag_fields { /* per member and call                        */
  const double *ub, *vb;            /* U(L,KSZU(L)), V(L,KSZV(L)): layer 1 here   */
  const double *vu, *uv;            /* VU, UV                                      */
  const double *h1u, *h1v;          /* H1U, H1V                                    */
  double *stbx, *stby;              /* out (optional): STBX, STBY                  */
  double *tbx, *tby;                /* out (optional): TBX, TBY                    */
} efdc_xm_drag_fields;
int32_t efdc_xm_bottom_stress_batch(efdc_xm_ctx *ctx, const efdc_xm_drag_params *prm,
                                    efdc_xm_drag_fields *f);

/* Explicit momentum producer: CALEXP2T's external-mode terms (calexp2t.f90:
 * 129-956 for IS2LMC = 0, ISVEG = 0, ISBODYF = 0, ISPNHYDS = 0, IATMP = 0,
 * ISWAVE < 2, ISCHAN /= 3): the upwind momentum fluxes FUHU, FVHU, FVHV, FUHV
 * (:202-237), the triangular-cell blocking STCUV (ITRICELL, :460-472), the
 * Coriolis-curvature coefficients CAC and their domain sum (:481-535), the
 * accelerations FCAX, FCAY (:545-562) with the type-2 open-boundary forms
 * (:605-645), the layer forcings FX, FY with the momentum of withdrawals and
 * sources FUHJ, FVHJ (:648-662), the flow-boundary edges (:664-689), the
 * horizontal momentum diffusion (ISHDMF >= 1, :797-811), and the depth sums
 * FCAXE, FCAYE, FXE, FYE (:940-956), on the device.  The sums stay on the
 * device for the next step: a step given FCAXE, FCAYE, FXE, FYE = NULL uses
 * them without an upload.  The internal-mode parts of CALEXP2T with KC > 1
 * (the vertical momentum fluxes FWU, FWV added to FX after the sums, :429-
 * 457 and :960-975, the buoyancy forcing and the shears DU, DV) stay with the
 * host's internal mode, which takes FX, FY, FCAX, FCAY per layer from here.
 * Layer arrays hold K = 1..kc at [(K-1)*ld + L-1] (ld = LCM for a Fortran
 * A(LCM,KCM)).  Cells outside the wet set hold 0 in every output, as the
 * reference's arrays of dry cells do (zeroed on drying, :131-175, and never
 * written while dry); the flow-boundary edges still apply to them.
 *
 * Static part, per member (efdc_xm_set_momentum): */
typedef struct efdc_xm_momentum {
  int32_t kc;                         /* KC (1..64)                                   */
  int32_t ld;                         /* leading dimension of the layer arrays (LCM)  */
  const double *fcorc, *dydi, *dxdj;  /* FCORC, DYDI, DXDJ (:489)                     */
  const double *scax, *scay;          /* SCAX, SCAY (:558-559)                        */
  const double *saax, *saay;          /* SAAX, SAAY (:668-688)                        */
  const double *sgzu, *sgzv;          /* SGZU(L,K), SGZV(L,K): layers (:944-947)      */
  const double *fsgzu, *fsgzv;        /* FSGZU(L,K), FSGZV(L,K): layers (:657-658)    */
  const double *stcuv;                /* STCUV (ITRICELL > 0) or NULL                 */
  const double *sdx, *sdy;            /* SDX, SDY (ISHDMF >= 1) or NULL               */
  const int32_t *lhdmf;               /* LHDMF(L,KC) as 0/1 (ISHDMF >= 1) or NULL     */
  const int32_t *lnwc, *lsec;         /* LNWC, LSEC: the NW and SE diagonal cells     */
  int32_t nbcs;                       /* NBCS: flow-boundary cells                    */
  int32_t pad_;
  const int32_t *lbcs, *lberc, *lbnrc; /* LBCS, LBERC, LBNRC [nbcs]                   */
} efdc_xm_momentum;
int32_t efdc_xm_set_momentum(efdc_xm_ctx *ctx, int32_t member, const efdc_xm_momentum *mo);

typedef struct efdc_xm_explicit_params { /* per member and call                    */
  double snlt;                        /* SNLT                                         */
  int32_t iscurvature;                /* ISCURVATURE                                  */
  int32_t ishdmf;                     /* ISHDMF                                       */
} efdc_xm_explicit_params;

typedef struct efdc_xm_explicit_fields { /* per member and call                    */
  const double *u, *v;                /* U(L,K), V(L,K) at entry: layers (these four
                                         NULL in every member: the previous call's)   */
  const double *uhdy, *vhdx;          /* UHDY(L,K), VHDX(L,K) at entry: layers        */
  const double *hp;                   /* HP                                           */
  const int32_t *wet;                 /* 0/1: the wet set LWET (LMASKDRY with ISDRY >
                                         0); NULL: every water cell                   */
  const double *fuhj, *fvhj;          /* FUHJ, FVHJ: layers (withdrawal/return and
                                         source momentum, :334-424) or NULL (zero)    */
  const double *fmdux, *fmduy;        /* ISHDMF >= 1: CALHDMF's FMDUX, FMDUY, FMDVX,  */
  const double *fmdvx, *fmdvy;        /*   FMDVY (layers)                             */
  double *fcaxe, *fcaye, *fxe, *fye;  /* out, or NULL (kept on the device)            */
  double *fcax, *fcay, *fx, *fy;      /* out: layers, or NULL                         */
  double *cac;                        /* out: layers, or NULL                         */
} efdc_xm_explicit_fields;

/* One call per time step, before the step that reads its sums (the order of
 * hdmt2t.f90:494-509).  Replaces CALL CALEXP2T for the options above (the
 * Fortran shim stops on the others); kc may differ by member. */
int32_t efdc_xm_explicit_batch(efdc_xm_ctx *ctx, const efdc_xm_explicit_params *prm,
                               efdc_xm_explicit_fields *f);

/* Standalone replacement of CONGRAD (congrad.f90:1-191) for callers that
 * assemble the scaled system themselves (e.g. calpuv9c.f90:446).  Arrays are
 * 1-based Fortran arrays as above; P is the initial guess and the result.
 * precision selects FP64 or MIXED.  *iters = ITER at exit (IDRYTBP). */
int32_t efdc_xm_congrad(efdc_xm_ctx *ctx, const double *ccc, const double *ccs,
                        const double *ccn, const double *ccw, const double *cce,
                        const double *ccci, const double *fptmp, double *p,
                        double rsqm, int32_t iterm, int32_t precision,
                        int32_t *iters, double *rsq);

/* ---- Ensembles: several independent basins in one context ----
 *
 * No counterpart in the reference, which runs one basin per process.  A
 * batch context holds `nmembers` basins ("members": ensemble runs,
 * calibration perturbations, or unrelated grids of any sizes) and advances
 * all of them with one launch sequence per step, each member exactly as
 * efdc_xm_step would advance it alone: every reduction (CCMNM, the PCG dot
 * products, the wet/dry re-solve flag, the negative-depth count) is taken per
 * member, each member stops its PCG at its own RSQM/ITERM and sweeps wet/dry
 * its own number of times.  All members must use the same `precision`.
 * Arrays of structures are indexed by member (grids[m], prm[m], f[m],
 * stats[m]); a field pointer is either given for every member or for none.
 * The return value is the first member error, else EFDC_XM_NEG_DEPTH if any
 * member had negative depths, else EFDC_XM_OK; stats[m].status is per member.
 * The single-basin functions above are the same code with one member and
 * refuse a context that holds more than one. */
efdc_xm_ctx *efdc_xm_create_batch(const efdc_xm_grid *grids, int32_t nmembers,
                                  int32_t device);
int32_t efdc_xm_nmembers(const efdc_xm_ctx *ctx);
int32_t efdc_xm_step_batch(efdc_xm_ctx *ctx, const efdc_xm_params *prm,
                           efdc_xm_fields *f, efdc_xm_stats *stats);
int32_t efdc_xm_upload_batch(efdc_xm_ctx *ctx, const efdc_xm_fields *f);
int32_t efdc_xm_step_device_batch(efdc_xm_ctx *ctx, const efdc_xm_params *prm,
                                  efdc_xm_stats *stats);
int32_t efdc_xm_download_batch(efdc_xm_ctx *ctx, efdc_xm_fields *f);

/* ---- Calibration: the reverse (adjoint) of the external mode ----
 *
 * No counterpart in the reference.  For single-basin contexts with clamped
 * open boundaries (ISPB=0), ISDRY=0, FP64.  The calibration model is
 * CALPUV2C preceded by a bottom drag written from a per-cell Manning n:
 * TBX = STBX*SQRT(VU^2+U^2)*U with STBX = G*n_u^2/HU^(1/3) (the form of
 * hdmt2t.f90:682 with AVCON1=0; U the depth-averaged u-face velocity, VU the
 * mean of the four v-face velocities around it, n_u the mean n of the face's
 * two cells), and TBY alike.  The adjoint of a step runs the step again from
 * a snapshot of its start state, then the reverse kernels, whose implicit
 * solve is a CG solve with the step's own (symmetric) operator.
 *
 * Typical use (N steps, a snapshot every K steps):
 *   forward:  snapshot(n/K) every K steps; calib_step(n); calib_gauges()
 *   backward: adjoint_reset(); for each K-step segment, last first: restore
 *             the segment's snapshot, rerun its steps taking one snapshot per
 *             step, then for each step n of the segment, last first:
 *             add_p_adjoint(d loss / d P after step n); adjoint_step(n)
 *   result:   calib_gradients()                                          */
int32_t efdc_xm_calib_enable(efdc_xm_ctx *ctx, int32_t nsnap); /* nsnap snapshot slots */
int32_t efdc_xm_calib_set_roughness(efdc_xm_ctx *ctx, const double *log_n); /* 1..LC */
/* harmonic amplitudes PCB/PSB of every open-boundary cell, packed in the
 * W, E, S, N order of the grid's lists: [cell*mtmax + m], mtmax = MTIDE */
int32_t efdc_xm_calib_set_harmonics(efdc_xm_ctx *ctx, const double *pcb, const double *psb);
int32_t efdc_xm_calib_snapshot(efdc_xm_ctx *ctx, int32_t slot); /* P, HP, HU, HV, UHDYE, VHDXE */
int32_t efdc_xm_calib_restore(efdc_xm_ctx *ctx, int32_t slot);
int32_t efdc_xm_calib_step(efdc_xm_ctx *ctx, const efdc_xm_params *prm, efdc_xm_stats *stats);
int32_t efdc_xm_calib_gauges(efdc_xm_ctx *ctx, int32_t n, const int32_t *l, double *p_out);
int32_t efdc_xm_calib_adjoint_reset(efdc_xm_ctx *ctx);
/* d(loss)/dP += w at cells l (P after the step whose adjoint runs next) */
int32_t efdc_xm_calib_add_p_adjoint(efdc_xm_ctx *ctx, int32_t n, const int32_t *l,
                                    const double *w);
/* the reverse of the step that starts at snapshot `slot`; the adjoint solve
 * stops at |r| <= rel_tol*|b| */
int32_t efdc_xm_calib_adjoint_step(efdc_xm_ctx *ctx, const efdc_xm_params *prm, int32_t slot,
                                   double rel_tol, int32_t *cg_iters);
/* accumulated d(loss)/d(log n) and d(loss)/d(BELV) (1..LC, elements 2..LA
 * written), d(loss)/d(PCB), d(loss)/d(PSB) (packed as above), and the
 * adjoint of the state at the start of the last reversed step (P, HP, HU,
 * HV, UHDYE, VHDXE; any may be NULL); *n_clamped counts boundary targets
 * that were dry-clamped (not differentiated) */
int32_t efdc_xm_calib_gradients(efdc_xm_ctx *ctx, double *dlog_n, double *dbelv, double *dpcb,
                                double *dpsb, double *const state[6], int32_t *n_clamped);

/* ---- Extensions with no counterpart in the reference (measurement hooks) ---- */

/* The CUDA stream (cudaStream_t) every call of this context runs on, so a
 * caller can order its own work or CUDA events against the solver. */
void *efdc_xm_stream(efdc_xm_ctx *ctx);

/* Number of kernels this library has launched in the process so far. */
int64_t efdc_xm_kernel_launches(void);

/* Schedule autotuner.  No counterpart in the reference, whose only schedule
 * rule is its thread count NOPTIMAL = MIN(NTHREADS,8,MAX(LA/100,1))
 * (calpuv2c.f90:61-62).  A schedule is the set of options above that change
 * the speed of a step but not its results (beyond the MIXED form's error
 * bar).  efdc_xm_autotune picks one for the context's workload: it looks the
 * workload's key up in the text file `table` and applies the schedule found
 * there (no measurement), or, when the key is absent or flags has
 * EFDC_XM_TUNE_MEASURE, times the solve of the system the last step assembled
 * (every member must have stepped once with `precision`; P is put back) under
 * candidate schedules -- one option at a time, candidates in a fixed order,
 * each the median of 5 timed solves, a candidate replacing the incumbent only
 * when 2 % faster -- applies the result and appends it to the table.  *solve_ms: the measured
 * solve time of the chosen schedule (0 when replayed).  The key holds the
 * precision, the floor log2 of the member count and of the water cells, and
 * whether the operator may be unsymmetric or has sub-grid channels. */
typedef struct efdc_xm_schedule {
  int32_t kernel_variant;  /* EFDC_XM_OPT_KERNEL_VARIANT */
  int32_t ctas_matvec;     /* EFDC_XM_OPT_CTAS_MATVEC */
  int32_t ctas_update;     /* EFDC_XM_OPT_CTAS_UPDATE */
  int32_t graph_iters;     /* EFDC_XM_OPT_GRAPH_ITERS */
  int32_t poly_threshold;  /* EFDC_XM_OPT_POLY_THRESHOLD */
  int32_t inner_margin;    /* EFDC_XM_OPT_INNER_MARGIN */
  int32_t inner_tol;       /* EFDC_XM_OPT_INNER_TOL */
} efdc_xm_schedule;
enum { EFDC_XM_TUNE_MEASURE = 1 };
int32_t efdc_xm_autotune(efdc_xm_ctx *ctx, int32_t precision, const char *table, int32_t flags,
                         efdc_xm_schedule *chosen, double *solve_ms);
/* The table key of a context's workload (NUL-terminated into buf). */
int32_t efdc_xm_tune_key(const efdc_xm_ctx *ctx, int32_t precision, char *buf, int32_t len);
/* The schedule `table` holds for `key` (its last line with that key);
 * EFDC_XM_BAD_ARGUMENT when there is none.  Reads the file only: no GPU. */
int32_t efdc_xm_tune_lookup(const char *table, const char *key, efdc_xm_schedule *out);

/* Number of times a step or solve call of this library has waited for the
 * device so far (host synchronisations).  A step whose loops run on the
 * device (EFDC_XM_OPT_DEVICE_LOOPS) waits once, when it has finished. */
int64_t efdc_xm_host_waits(void);

/* Options of a context (no counterpart in the reference).
 *   EFDC_XM_OPT_DEVICE_LOOPS (default 1): 1 runs each step as one CUDA graph
 *     whose data-dependent loops -- the CG iterations (congrad.f90:91-169),
 *     the MIXED refinement passes and the wet/dry re-solves (the GOTO 1000
 *     of calpuv2c.f90:597-601, 726-749) -- are conditional nodes decided on
 *     the device, so the host waits once per step; 0 drives those loops from
 *     the host, polling the device between groups of iterations.  Both run
 *     the same kernels in the same order.
 *   EFDC_XM_OPT_GRAPH_ITERS (default 4, 1..32): CG iterations per loop body.
 *   EFDC_XM_OPT_KERNEL_VARIANT (default 0): the MIXED inner iteration's
 *     kernels; 0 fetches each 4-tile unit's descriptors (its member's values,
 *     its tiles' neighbours) one unit ahead, 1 fetches them for 32 units at a
 *     time into shared memory, 2 does that and also stages each unit's rows
 *     in shared memory with bulk copies issued one unit ahead, 3 fetches them
 *     as 1 does and issues every load of a row before the row's first
 *     dependent operation (at fewer CTAs per SM).  All give the same results
 *     bit for bit.
 *   EFDC_XM_OPT_CTAS_MATVEC, EFDC_XM_OPT_CTAS_UPDATE (default 0, 0..32): with
 *     variants 1, 2 and 3, caps on the resident CTAs per SM of the inner
 *     iteration's matrix-vector and update kernels (0: as many as fit).
 *   EFDC_XM_OPT_POLY_THRESHOLD (default 10, 0..100000): a MIXED member whose
 *     last solve took more than this many Jacobi-equivalent inner iterations
 *     uses the polynomial preconditioner (0: always, 100000: never).
 *   EFDC_XM_OPT_INNER_MARGIN (default 0, 0..6): the MIXED inner solve reduces
 *     its residual 10^value times further than the FP64 residual needs to
 *     reach its stop, trading inner iterations for refinement passes.
 *   EFDC_XM_OPT_INNER_TOL (default 60, 40..75): a MIXED inner solve reduces
 *     its residual by at least 10^(-value/10) in norm before the next FP64
 *     refinement pass, where the FP64 stop needs more than that.
 *   EFDC_XM_OPT_SMALL_SOLVE (default 1): 1 runs the FP64 CG of contexts
 *     whose members are all small (up to about 4,000 slots of 32x8 tiles,
 *     e.g. basins of a few thousand cells) and have no sub-grid channels as
 *     one launch with one CTA per member, its vectors in shared memory; 0
 *     runs it as the kernels of every other context.  Both give the same
 *     results bit for bit.
 *   EFDC_XM_OPT_FOLD_REDUCE (default 1, 0..2): 2 finishes each member's CG
 *     sums (its dot products, ALPHA, BETA and stop tests) inside the kernel
 *     that forms them, in the CTA that stores the member's last partial sum;
 *     0 runs a separate member-reduce kernel after each CG kernel; 1 takes
 *     the first form for contexts of up to 4 members and the second for
 *     larger batches.  Contexts with sub-grid channels always take the
 *     second form.  Both give the same results bit for bit.
 *   EFDC_XM_OPT_CHUNKS (default 8, 1..32): efdc_xm_step_batch of two or
 *     more members steps them in this many member chunks of about equal cell
 *     counts, so that the upload of one chunk, the step of an earlier one and
 *     the download of a still earlier one overlap.  Results do not depend on
 *     it.
 * Results stay within the MIXED form's error bar whatever the schedule; the
 * FP64 form's results do not depend on it.
 * Returns EFDC_XM_BAD_ARGUMENT for an unknown option or value. */
enum {
  EFDC_XM_OPT_DEVICE_LOOPS = 1,
  EFDC_XM_OPT_GRAPH_ITERS = 2,
  EFDC_XM_OPT_KERNEL_VARIANT = 3,
  EFDC_XM_OPT_CTAS_MATVEC = 4,
  EFDC_XM_OPT_CTAS_UPDATE = 5,
  EFDC_XM_OPT_POLY_THRESHOLD = 6,
  EFDC_XM_OPT_INNER_MARGIN = 7,
  EFDC_XM_OPT_INNER_TOL = 8,
  EFDC_XM_OPT_SMALL_SOLVE = 9,
  EFDC_XM_OPT_FOLD_REDUCE = 10,
  EFDC_XM_OPT_CHUNKS = 11
};
int32_t efdc_xm_set_option(efdc_xm_ctx *ctx, int32_t option, int32_t value);

/* Bytes copied host->device (*h2d) and device->host (*d2h) by the upload,
 * download and step calls of every context since the library was loaded
 * (the caller's arrays only: no small control transfers). */
void efdc_xm_transfer_bytes(int64_t *h2d, int64_t *d2h);

/* Average device time (CUDA events on the context's stream) of the CG
 * iteration kernels on the system currently assembled in the context:
 * `reps` matrix-vector (p update + A*p + p.Ap) and update (x, r, r.z, r.r)
 * launches of the given precision.  Leaves P unchanged. */
typedef struct efdc_xm_ktime {
  double ms_matvec;     /* per launch */
  double ms_update;     /* per launch */
  int32_t reps;
  int32_t ncells;       /* water cells, LA-1 summed over members */
  int32_t nslots;       /* tile slots processed per launch (incl. land padding) */
  int32_t ncells_poly;  /* MIXED: water cells of the members whose inner solve uses the
                         * polynomial preconditioner (their update moves 36 B per cell,
                         * the others' 24 B) */
} efdc_xm_ktime;
int32_t efdc_xm_time_kernels(efdc_xm_ctx *ctx, int32_t precision, int32_t reps,
                             efdc_xm_ktime *out);

/* ---- Entry point with no counterpart in the reference ----
 *
 * CONGRAD that allocates nothing.  For callers that cannot let this library
 * allocate GPU memory: a host code that gives all of its device memory to its
 * own pool or budget, a time-critical loop where an allocation could stall or
 * fail, or a caller whose data already sit in device arrays it manages (CUDA
 * Fortran device arrays, a framework's tensors).  It solves the same system
 * as efdc_xm_congrad (congrad.f90:54-187, FP64, CCCI recomputed as 1/CCC) on
 * the reference's own layout, without a context:
 *   - every array is a DEVICE pointer to a 1-based Fortran-layout array
 *     (element L at [L-1], L = 1..LC with LC = LA+1); P is the initial guess
 *     and receives the result; iters and rsq are host pointers;
 *   - the solver's vectors live in one fixed array of device memory declared
 *     at file scope in the library, sized for at most
 *     EFDC_XM_NOALLOC_MAX_CELLS water cells (12.6 MB); every GPU that loads
 *     the library holds it until the process exits.  Larger LA is rejected
 *     with EFDC_XM_BAD_ARGUMENT and a message (efdc_xm_last_error);
 *   - the first call on a device looks up that array's device address (with
 *     that device current) and keeps it;
 *   - all calls share the array: calls that overlap on the GPU (other
 *     streams, other host threads) race; the call returns after its work on
 *     `stream` (a cudaStream_t, NULL = legacy default stream) finished;
 *   - every call reads its stop test back to the host: it copies the control
 *     block to host memory and synchronizes `stream` after every 8
 *     iterations, so it must not be called while a stream capture is active
 *     (on `stream` or, in global capture mode, anywhere in the process). */
#define EFDC_XM_NOALLOC_MAX_CELLS 524288
int32_t efdc_xm_congrad_noalloc(int32_t la, const int32_t *lnc, const int32_t *lsc,
                                const int32_t *lec, const int32_t *lwc, const double *ccc,
                                const double *ccs, const double *ccn, const double *ccw,
                                const double *cce, const double *fptmp, double *p, double rsqm,
                                int32_t iterm, void *stream, int32_t *iters, double *rsq);

#ifdef __cplusplus
}
#endif

#endif /* EFDC_XM_H */
