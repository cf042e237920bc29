// xm_internal.h -- device data layout and kernel interface of libefdc_xm.
//
// Layout ("bricks"): each basin's structured grid is cut into 32x8-cell
// tiles.  Tiles holding at least one water cell are stored contiguously,
// member after member, each member's tiles ordered along a Morton (Z) curve of
// their tile coordinates and preceded by the member's ghost tile (all land);
// inside a tile a cell's slot is ty*32+tx.  Slot d = tile*256 + ty*32 + tx.
// Tile 0 is member 0's ghost tile.  Neighbours
// come from the slot position plus a 4-entry tile neighbour table, so no
// per-cell index arrays are read in the solver: E/W neighbours are adjacent
// words and N/S neighbours are the rows above and below, which keeps every
// warp access a contiguous 32-cell row.
//
// A context holds M >= 1 independent basins ("members" of an ensemble); one
// launch of each kernel covers all of them.  Everything that the reference
// reduces over a basin (CCMNM, the CG dot products, the wet/dry re-solve flag,
// the negative-depth count) is reduced per member.
//
// Land slots (padding inside a tile, and the member's ghost tile, which a
// missing neighbour tile maps to) stand for EFDC+'s ghost cell LC (a missing
// neighbour maps to LC, EFDC/cellmap.f90:80-134): they hold the member's
// element-LC values and are never written by the solver.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace xm {

constexpr int TX = 32;
constexpr int TY = 8;
constexpr int TILE = TX * TY;  // 256 slots per tile
constexpr int NT = TILE;       // threads per CTA in the cell kernels
constexpr int MT_MAX = 16;     // max harmonic constituents per call

// CHAN: a water cell that is the host or guest of a sub-grid channel (its CC
// enters the minimum diagonal after the channel terms, not in the assembly)
enum SlotKind : uint8_t { LAND = 0, WATER = 1, OPENBC = 2, CHAN = 3 };

// Per-member scalars of one call (device memory, refreshed every step).
struct StepScalars {
  double delt, deltd2, delti, g, gi, hdry, rsqm, snlt, ritb1;
  int isdry, ndrystp, isbal, iterm;
  int max_sweeps;       // wet/dry re-solve cap (the reference's 500)
  int pad_sc;
  double rlamn;         // QCHERR: implicit weight of the channel flows
  int chan_consistent;  // channels: 1 = A*p with -CCCCHH (else as congradc.f90 writes it)
  int baro;             // BSC > 1e-6: the baroclinic terms FPGXE, FPGYE enter
  double gp;            // GP
  int istl;             // 0: CALPUV2C; 3 or 2: CALPUV9C(ISTL_) (the same for every member)
  int nctbc;            // NCTBC (CALPUV9C, ISTL_ = 3: 1 halves UHDYE, VHDXE on advancing)
  double rold, rnew;    // ROLD, RNEW: blend of FPGXE, FPGYE (CALPUV9C)
  int isitb, isveg;     // ISITB >= 1: implicit bottom drag; ISVEG > 0: vegetation drag
  double ritb;          // RITB
  double cosv[MT_MAX], sinv[MT_MAX];
};

// Device-side control block of one member.  Written by the "last CTA" of a
// member's reductions; read by the host once per solve.
struct Ctl {
  double rpcg, alpha, beta, rsq, papcg;
  double rsq64, rsq_target;       // MIXED: outer residual, inner target
  double ccmnm_int, ccmnm_bc;     // min CC over interior / open-BC cells (atomic min on bits)
  int iter, done, status, parity; // status: enum efdc_xm_status
  int inner_iter, outer, idone;   // MIXED bookkeeping (idone: inner solve finished)
  int asym;                       // 1 if the scaled operator is not symmetric (2: unexpected)
  int icordry;                    // wet/dry re-solve flag of this sweep
  int active;                     // member takes part in the current sweep
  int nneg, nnonfinite, nwasted;
  unsigned int counter;           // last-CTA arrival counter
  // the member's step, summed over its sweeps where the sweep loop runs on
  // the device (k_after_solve, k_sweep_next); zero at the start of a step
  int stepping;                   // the member takes part in this step
  int mstatus;                    // its status (enum efdc_xm_status)
  int sweep;                      // re-solves so far (NCORDRY)
  int solves, iters_total, iters_last, outer_total;
  int inner_first;                // MIXED: inner iterations of the first pass of the last solve
  int last_inner;                 // MIXED: inner iterations of the last pass that had some
  int pad;
  double rsq_last, ccmnm_last;
};

// Loops of a step whose control runs on the device (conditional graph
// nodes): the CG iterations, the MIXED outer passes and inner iterations, and
// the wet/dry sweeps.
enum Loop : int { LOOP_CG = 0, LOOP_OUTER = 1, LOOP_INNER = 2, LOOP_SWEEP = 3, NLOOP = 4 };

// Counters across members, polled by the host (or read by the loop-control
// kernels of a device-driven step).
struct Glob {
  int ndone;     // members whose solve finished
  int nidone;    // members whose inner (FP32) solve finished
  int nicordry;  // members that need another wet/dry sweep
  int err;       // nonzero: a bounded device-side wait ran out (a timeout status)
  int loop[NLOOP];  // body executions of the loop now running (each loop's cap)
  int tot[NLOOP];   // body executions in the step (the launch count)
};

// Static per-slot model data (FP64).  Land slots hold element LC.
// Sub-grid channels of all members, packed member after member (channel NMD
// of member m at cstart[m] + NMD - 1).  Slots are tile-order cells.
struct DevChan {
  int n;                     // channels of all members (0: none)
  const int *cstart;         // [M+1]
  const int *type;           // MDCHTYP: 1 x-direction, 2 y-direction
  const int *host, *guest;   // slots of LMDCHH and of LMDCHU (x) / LMDCHV (y)
  const int *gu;             // slot of LMDCHU for the y-direction HP test; -1: L = 1
  const int *qhost, *qguest; // quads holding the host / guest slot
  const int *first_host, *first_guest;  // 1: first endpoint of the member on its cell
  const double *len, *fric;  // CHANLEN, CHANFRIC
  const double *gw, *gl;     // guest's WCHAN (DXP x, DYP y) and cross length (DYP x, DXP y)
  const double *hp1;         // [M] HP(1) of each member (its value at upload)
  double *qu, *qv, *qun, *qvn;  // QCHANU, QCHANV, QCHANUN, QCHANVN
  double *qut, *qvt;         // QCHANUT, QCHANVT: the flows at step entry
  double *cu, *cv, *chh;     // CCCCHU, CCCCHV, CCCCHH (unscaled)
  double *p1h, *p1g;         // P1 at host and guest (P at step entry)
  double *p0h, *p0g;         // P at the entry of a MIXED solve
  float *hh32;               // MIXED: coupling of the Jacobi-scaled FP32 operator
  int *iact;                 // IACTIVE
};

// Baroclinic terms (CALEBI, standard sigma grid): layer planes of `stride`
// elements (layer K at [(K-1)*stride]) in tile order.
struct DevBaro {
  int kc;                  // layers (0: not set)
  long long stride;        // elements per plane (the slot count)
  const double *dzc, *zz;  // DZC(L,K), ZZ(L,K)
  double *b;               // B(L,K), uploaded with the fields
  double *bi1, *bi2, *be;  // BI1W=BI1S, BI2W=BI2S, BEW=BES: kept between steps
};

struct DevStatic {
  const int4 *tnbr;       // [ntile] (w, e, s, n) neighbour tiles (missing: the member's ghost tile)
  const uint8_t *kind;    // [nslot]
  const int *lidx;        // [nslot] member-local L of the slot, 0 for land
  const int *tile_member; // [ntile] member of each tile
  const int4 *quads;      // [nquad] (member, first tile, tiles of the member in it (1..4), 0):
                          // the 4-tile units of the CG kernels
  const int *qstart;      // [M+1] first quad of each member
  const int *tend;        // [M] one past the member's last tile
  const StepScalars *sc;  // [M] per-member scalars of the current step
  int nquad;
  int nmember;
  const double *dxyp, *dxyip, *dxiu, *dyiu, *dxiv, *dyiv, *dxyu, *dxyv;
  const double *hruo, *hrvo, *subo, *svbo, *sbxo, *sbyo, *belv;
  const double *fsgzu, *fsgzv;  // 0.5/DXYU, 0.5/DXYV (calpuv2c.f90:111-116)
  DevChan ch;                   // sub-grid channels (ch.n == 0: none)
  DevBaro baro;                 // layers and buoyancy integrals (baro.kc == 0: none)
};

// Per-step state and work arrays (tile layout).
struct DevState {
  double *p, *hp, *h1p, *hu, *hv, *uhdye, *vhdxe, *sub, *svb, *sbx, *sby;
  int *lmaskdry, *iscdry, *lopenbcdry, *natdry, *oldmask;
  const double *fcaxe, *fcaye, *fxe, *fye, *tsx, *tsy, *tbx, *tby, *qsume;
  double *uhe, *vhe, *hpi, *hui, *hvi, *qdwaste, *vdwaste;
  double *uhdy1e, *vhdx1e, *sub1, *svb1, *fp1, *fuhdye, *fvhdxe;
  double *fp, *cc, *cs, *cw, *ce, *cn;  // unscaled system (FP64)
  // wet/dry scratch: decision codes and the new face switches of a sweep
  int *wd_act;
  double *sub_n, *svb_n, *sbx_n, *sby_n;
  int *wasted;  // 1 where NDRYSTP volume wasting fired this step
  // three time levels (CALPUV9C), allocated on first use: P1, H2P, UHDY2E,
  // VHDX2E, H1U, H1V, HUTMP, HVTMP, FPGXE, FPGYE and the level n-1 stresses
  double *p1, *h2p, *uhdy2e, *vhdx2e, *h1u, *h1v, *hutmp, *hvtmp, *fpgxe, *fpgye;
  const double *tsx1, *tsy1, *tbx1, *tby1;
  // views of the step being taken, set by the host before its first kernel:
  // huc, hvc: the face depths of the coefficients (HU, HV; HUTMP, HVTMP in
  //   CALPUV9C(2));
  // hb, ub, vb: the level the continuity starts from and its transports
  //   (H1P, UHDY1E, VHDX1E; H2P, UHDY2E, VHDX2E in CALPUV9C(3)); hb is also
  //   HPPMC of the drying checks;
  // hp0: HP at entry (the H1P buffer after the time-level advance; HP in
  //   CALPUV9C(2), which does not advance).
  const double *huc, *hvc, *hb, *ub, *vb, *hp0;
  // RCX, RCY: the implicit drag coefficients of the faces (calpuv2c.f90:
  // 222-243), 1 on water and 0 on land slots until a step with ISITB >= 1 or
  // ISVEG > 0 sets them; kept between steps like the reference's module arrays
  double *rcx, *rcy;
  // the implicit drag's inputs (allocated by the first upload that carries
  // them): U(L,KSZU(L)), V(L,KSZV(L)), VU, UV, STBX, STBY, FXVEGE, FYVEGE
  const double *ubot, *vbot, *vu, *uv, *stbx, *stby, *fxvege, *fyvege;
};

// Scaled system and CG vectors.
struct DevSystem {
  double *ccc, *ccs, *ccw, *cce, *ccn, *fptmp;  // FP64 scaled coefficients, b
  double *r, *pa, *pb, *ap;                      // FP64 CG vectors (p double-buffered)
  double *z;                                     // FP64: z = CCCI*r, written with r
  // MIXED: the FP32 inner system is the Jacobi-scaled operator
  // Ahat = D^-1/2 A D^-1/2 (unit diagonal, D = CCC), so CG on it equals
  // Jacobi-PCG on A and needs no diagonal array:
  float *as32, *aw32, *ae32, *an32;              // off-diagonals of Ahat (E/N only if unsymmetric)
  float *r32, *pa32, *pb32, *ap32, *x32;         // FP32 inner CG vectors (scaled)
  float *z32;                                    // preconditioned residual z = M^-1 r
  float *r32b;                                   // second residual buffer (r32 / r32b by parity)
  const int *mpoly;                              // [M] 1: Neumann polynomial, 0: Jacobi (per solve)
  int *err;                                      // Glob::err of the context
};

// The system a MIXED solve refines: a step's unscaled assembly (FP, CC, CS,
// CW, CE, CN), or a caller's scaled system (standalone CONGRAD).  The inner
// operator D^-1/2 A D^-1/2 and the correction D^-1/2 x do not depend on the
// scaling; only RSQ (taken on the scaled system, as CONGRAD's) does.
struct SysView {
  const double *fp, *cc, *cs, *cw, *ce, *cn;
  int unscaled;  // 1: RSQ = sum(r^2) / CCMNM^2
};

// Bottom-stress producer (CALTBXY's drag coefficients and the bottom stresses
// TBX, TBY): the static bed of the members that have one, the drag
// coefficients kept between calls, and each call's internal-mode inputs, in
// tile order.
struct DevBed {
  const double *zbr, *zbratu, *zbratv, *sgzuu, *sgzvv, *stbxo, *stbyo;
  double *stbx, *stby;                      // STBX, STBY (0 before the first call)
  double *ub, *vb, *vu, *uv, *h1u, *h1v;    // U, V of the bottom layer, VU, UV, H1U, H1V
};

// Explicit momentum producer (CALEXP2T's external-mode terms): per-member
// scalars of one call, and the device arrays in tile order.  Layer arrays
// are [k][slot] with stride ls; per-slot int arrays hold 0/1 or slots.
struct MomScalars {
  double snlt;  // SNLT
  int kc;       // layers of the member
  int on;       // the member takes part (it has its static part)
  int curv;     // ISCURVATURE
  int tri;      // STCUV given (ITRICELL > 0)
  int hdmf;     // ISHDMF >= 1
  int fuhj;     // FUHJ, FVHJ given
};

struct MomDev {
  const double *fcorc, *dydi, *dxdj, *scax, *scay, *saax, *saay, *stcuv, *sdx, *sdy;
  const int *lhdmf;   // LHDMF as 0/1
  const int *nw, *se; // slots of LNWC(L), LSEC(L) (the member's ghost slot for LC)
  const double *sgzu, *sgzv, *fsgzu, *fsgzv;                   // static layers
  const double *u, *v, *uhdy, *vhdx, *fuhj, *fvhj;             // per-call layers
  const double *fmdux, *fmduy, *fmdvx, *fmdvy;
  const double *hp;   // HP of the call (the step's HP when the caller gives none)
  const int *wet;     // the wet set as 0/1
  double *fuhu, *fvhu, *fvhv, *fuhv, *cac;                      // work layers
  double *fcax, *fcay, *fx, *fy;                                // output layers
  double *cacsum;     // [M] the members' sums of CAC
  const MomScalars *sc;
  const int4 *t2, *bc;            // the serial lists (see k_mom_edges)
  const int *t2start, *bcstart;   // [M+1]
  size_t ls;                      // layer stride (slots)
};

// Per-member scalars of one bottom-stress call.
struct DragScalars {
  double delt, avcon1, avcon, vismud, visfac;
  int isdry, n, ntstbc;
  int kc1;  // KC = 1: the single-layer form of the rough drag
  int on;   // the member takes part (it has a bed)
  int pad;
};

// Open-boundary cells (packed per member: W, E, S, N in the reference's loop order).
struct DevObc {
  int n;                 // total number of open-boundary cells
  int mtmax;             // stride of pcb/psb (max MTIDE over members)
  const int *slot;       // [n] slot of the boundary cell
  const int *nbr;        // [n] slot of its interior neighbour (LEC/LWC/LNC/LSC)
  const int *side;       // [n] 0 W, 1 E, 2 S, 3 N
  const int *ispb;       // [n]
  const int *member;     // [n]
  const int *mtide;      // [M] harmonic constituents of each member
  const int *bstart;     // [M+1] first boundary cell of each member
  const double *pcb, *psb;  // [n*mtmax], index k*mtmax+m
  const double *pser;    // [n] per-step series part
};

// Calibration (adjoint) state of a single-member context, tile layout.
// "0" arrays are the step-start state (a snapshot), `psol` the step's CG
// solution P'; the adjoint arrays hold d(loss)/d(x).  in: adjoints of the
// step's outputs; out: of its inputs.
struct DevCalib {
  double *kappa;                                   // log Manning n per slot
  double *tbx, *tby;                               // the drag written for the step
  const double *p0, *hp0, *hu0, *hv0, *u0, *v0;    // P, HP, HU, HV, UHDYE, VHDXE at step start
  const double *psol;                              // P' (CG solution of the step)
  double *ap_in, *ahp_in, *ahu_in, *ahv_in, *au_in, *av_in;
  double *ap_out, *ahp_out, *ahu_out, *ahv_out, *au_out, *av_out;
  double *ahpe;            // adjoint of HP' (continuity output) after the face-depth terms
  double *rhs, *lam;       // adjoint solve: A lam = rhs
  double *afp, *afu, *afv; // adjoints of FP, FUHDYE, FVHDXE
  double *atbx, *atby;     // adjoints of TBX, TBY
  double *nbu, *nbv;       // adjoints of the face Manning n (u, v faces)
  double *vub, *uvb;       // adjoints of VU (at u faces) and UV (at v faces)
  double *akappa, *abelv;  // accumulated gradients w.r.t. log n and BELV
  double *apcb, *apsb;     // accumulated gradients w.r.t. PCB, PSB ([n_obc * mtmax])
  int *nflag;              // [1] boundary cells whose dry-clamp branch fired (not differentiated)
};

}  // namespace xm
