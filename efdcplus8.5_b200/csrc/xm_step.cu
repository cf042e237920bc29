// xm_step.cu -- FP64 kernels of one external-mode step (everything except the
// FP32 inner solve).  Compiled with -fmad=false: every statement rounds as
// the reference's SSE2 ReleaseDP64 build does (no fused multiply-add), so the
// per-cell arithmetic matches EFDC+ statement by statement; only the order of
// the global dot products differs (fixed-order tree instead of serial).
//
// The cell kernels are grid-stride loops over tiles (one 256-thread CTA
// processes a whole 32x8 tile per pass; tile 0, member 0's ghost tile, is
// skipped, and the other members' ghost tiles hold land slots only).  A tile
// belongs to one member of the ensemble; the member's scalars come from
// S.sc[m] and its reductions go to ctl[m].  `act[m]` says whether member m
// takes part in the current wet/dry sweep (or, for the finalisation kernels,
// whether its step is to be finalised).

#include <map>
#include <mutex>
#include <type_traits>

#include "xm_cg.cuh"
#include "xm_kernels.h"

namespace xm {

#define TILE_LOOP(ntile) for (int tile = blockIdx.x + 1; tile < (ntile); tile += gridDim.x)

#define TILE_MEMBER(S)                  \
  const int m = (S).tile_member[tile]; \
  const StepScalars &c = (S).sc[m]

// ---------------------------------------------------------------------------
// calpuv2c.f90:214-220: the explicit transports FUHDYE (face between cell d
// and its west neighbour, elevations P and PW) and FVHDXE (south face).
// UH1: UHDYE at entry (UHDY1E in CALPUV9C), HC: the face depth (HUTMP in
// CALPUV9C), TS, TB: the stresses (TSX1, TBX1 in CALPUV9C, calpuv9c.f90:216-217);
// FPGXE / FPGYE: the baroclinic terms, 0.0 without them.
__device__ __forceinline__ double fuh_face(const DevStatic &S, const DevState &X,
                                           const StepScalars &c, int d, double UH1, double HC,
                                           double P, double PW, double sub, double FPGXE,
                                           double TS, double TB) {
  return UH1 - c.deltd2 * sub * S.hruo[d] * HC * (P - PW) +
         sub * c.delt * S.dxiu[d] *
             (S.dxyu[d] * (TS - c.ritb1 * TB) + X.fcaxe[d] + FPGXE - c.snlt * X.fxe[d]);
}
__device__ __forceinline__ double fvh_face(const DevStatic &S, const DevState &X,
                                           const StepScalars &c, int d, double VH1, double HC,
                                           double P, double PS, double svb, double FPGYE,
                                           double TS, double TB) {
  return VH1 - c.deltd2 * svb * S.hrvo[d] * HC * (P - PS) +
         svb * c.delt * S.dyiv[d] *
             (S.dxyv[d] * (TS - c.ritb1 * TB) - X.fcaye[d] + FPGYE - c.snlt * X.fye[d]);
}

// calpuv2c.f90:192-201 (calpuv9c.f90:175-181): the external density
// gradients of the west and south faces of cell q.d from HP, HU, HV, SBX, SBY.
__device__ __forceinline__ void baro_faces(const DevStatic &S, const DevState &X,
                                           const StepScalars &c, const Nb &q, const double *HP,
                                           double &FPGXE, double &FPGYE) {
  const DevBaro &Bc = S.baro;
  const int d = q.d;
  FPGXE = -X.sbx[d] * X.hu[d] * c.gp *
          ((Bc.bi2[d] + Bc.bi2[q.w]) * (HP[d] - HP[q.w]) +
           2.0 * X.hu[d] * (Bc.bi1[d] - Bc.bi1[q.w]) +
           (Bc.be[d] + Bc.be[q.w]) * (S.belv[d] - S.belv[q.w]));
  FPGYE = -X.sby[d] * X.hv[d] * c.gp *
          ((Bc.bi2[d] + Bc.bi2[q.s]) * (HP[d] - HP[q.s]) +
           2.0 * X.hv[d] * (Bc.bi1[d] - Bc.bi1[q.s]) +
           (Bc.be[d] + Bc.be[q.s]) * (S.belv[d] - S.belv[q.s]));
}

// CALEBI (calebi.f90:73-120) for the standard sigma grid (KSZ = 1): the
// external buoyancy integrals of each wet cell (LWET of the last step: every
// cell with ISDRY = 0, else the cells with LMASKDRY).  The reference's two
// loops from the top layer down are one here (the same additions in the same
// order).
__global__ void __launch_bounds__(NT) k_calebi(DevStatic S, DevState X, int ntile,
                                              const int *act) {
  const DevBaro &Bc = S.baro;
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!c.baro || !act[m]) continue;
    const int d = tile * TILE + threadIdx.x;
    if (S.kind[d] == LAND) continue;
    if (c.isdry > 0 && !X.lmaskdry[d]) continue;
    double DBK = 0., BEC = 0., BI1C = 0., BI2C = 0.;
    for (int k = Bc.kc - 1; k >= 0; --k) {
      const size_t o = size_t(k) * size_t(Bc.stride) + d;
      const double DZCC = Bc.dzc[o];
      const double DZCB = DZCC * Bc.b[o];
      DBK = DBK + DZCB;
      const double BK = DBK - 0.5 * DZCB;
      BEC = BEC + DZCB;
      const double DZCBK = DZCC * BK;
      BI1C = BI1C + DZCBK;
      BI2C = BI2C + DZCBK + Bc.zz[o] * DZCB;
    }
    Bc.bi1[d] = BI1C;
    Bc.bi2[d] = BI2C;
    Bc.be[d] = BEC;
  }
}

// RCX (u face of slot x) and RCY (v face): the implicit-drag factors of a
// member with ISITB >= 1 or ISVEG > 0 (k_implicit_drag), else 1.0 without a
// load (calpuv2c.f90:97-102: RCX = RCY = 1 on water cells; a land slot's 0
// only ever multiplies its own zero switch SUB(LC) = SVB(LC) = 0, so 1.0 gives
// the same product there).
__device__ __forceinline__ bool has_drag(const StepScalars &c) {
  return c.isitb >= 1 || c.isveg > 0;
}
__device__ __forceinline__ double rc_x(const DevState &X, const StepScalars &c, int x) {
  return has_drag(c) ? X.rcx[x] : 1.0;
}
__device__ __forceinline__ double rc_y(const DevState &X, const StepScalars &c, int x) {
  return has_drag(c) ? X.rcy[x] : 1.0;
}

// calpuv2c.f90:282-290 (calpuv9c.f90:277, from P1, UHDY1E, VHDX1E); U, V: the
// transports at entry
__device__ __forceinline__ double fp1_cell(const DevStatic &S, const StepScalars &c,
                                           const Nb &q, double P, const double *U,
                                           const double *V) {
  const double C1 = 0.5 * c.g;
  return c.delti * S.dxyp[q.d] * P - C1 * (U[q.e] - U[q.d] + V[q.n] - V[q.d]);
}

// calpuv2c.f90:306-344 for cell q.d from its faces' transports: FP, CS, CW,
// CE, CN, CC.  Returns CC.
__device__ __forceinline__ double assemble_cell(const DevStatic &S, const DevState &X,
                                                const StepScalars &c, const Nb &q, double fp1,
                                                double fuh, double fuhe, double fvh,
                                                double fvhn) {
  const int d = q.d;
  // the loads first (the stores below could alias them for the compiler)
  const double sub = X.sub[d], svb = X.svb[d], sube = X.sub[q.e], svbn = X.svb[q.n];
  const double qsume = X.qsume[d], dxyp = S.dxyp[d];
  const double hrvo = S.hrvo[d], hruo = S.hruo[d], hruoe = S.hruo[q.e], hrvon = S.hrvo[q.n];
  const double hvc = X.hvc[d], huc = X.huc[d], huce = X.huc[q.e], hvcn = X.hvc[q.n];
  const double ry = rc_y(X, c, d), rx = rc_x(X, c, d), rxe = rc_x(X, c, q.e),
               ryn = rc_y(X, c, q.n);
  double C1 = 0.5 * c.g;
  X.fp[d] = fp1 - C1 * (sube * fuhe - sub * fuh + svbn * fvhn - svb * fvh - 2.0 * qsume);
  C1 = -0.5 * c.deltd2 * c.g;
  const double cs = C1 * svb * hrvo * ry * hvc;
  const double cw = C1 * sub * hruo * rx * huc;
  const double ce = C1 * sube * hruoe * rxe * huce;
  const double cn = C1 * svbn * hrvon * ryn * hvcn;
  const double cc = c.delti * dxyp - cs - cw - ce - cn;
  X.cs[d] = cs;
  X.cw[d] = cw;
  X.ce[d] = ce;
  X.cn[d] = cn;
  X.cc[d] = cc;
  return cc;
}

// ---------------------------------------------------------------------------
// calpuv2c.f90:164-293: switches, explicit transports, FP1.  The time-level
// advance of the 2D arrays this library owns (UHDY1E=UHDYE, VHDX1E=VHDXE,
// H1P=HP, :256-264) is either a buffer swap by the host before this kernel,
// when every member steps (COPY = false: the *1 buffers hold the entry
// values), or per-cell copies here (COPY = true: the entry values are in
// UHDYE, VHDXE, HP), which lets a subset of the members step (act).
// BARO: a member of the batch has baroclinic terms.  Each instance runs on a
// grid of its own occupancy (cell_grid).
constexpr int BEGIN_CTAS = 6;  // CTAs per SM the instance without BARO is held to (40 registers, no spills)
template <bool BARO, bool COPY>
__global__ void __launch_bounds__(NT, BARO ? 4 : BEGIN_CTAS) k_begin(DevStatic S, DevState X, int ntile,
                                                           const int *act) {
#define UE (COPY ? X.uhdye : X.uhdy1e)
#define VE (COPY ? X.vhdxe : X.vhdx1e)
#define HE (COPY ? X.hp : X.h1p)
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m]) continue;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    // every result first, the stores after (a store before a load would keep
    // the compiler from issuing the load early: the arrays could alias)
    const double sub = X.sub[d], svb = X.svb[d];
    const double P = X.p[d];
    double FPGXE = 0., FPGYE = 0.;
    if (BARO && c.baro)  // :192-201 (entry HP, HU, HV, SBX, SBY)
      baro_faces(S, X, c, q, HE, FPGXE, FPGYE);
    const double uh = UE[d], vh = VE[d];
    const double fuh =
        fuh_face(S, X, c, d, uh, X.hu[d], P, X.p[q.w], sub, FPGXE, X.tsx[d], X.tbx[d]);
    const double fvh =
        fvh_face(S, X, c, d, vh, X.hv[d], P, X.p[q.s], svb, FPGYE, X.tsy[d], X.tby[d]);
    const double fp1 = fp1_cell(S, c, q, P, UE, VE);
    if (c.isdry > 0) {  // :172-190
      X.iscdry[d] = 0;
      X.sub1[d] = sub;
      X.svb1[d] = svb;
      X.oldmask[d] = X.lmaskdry[d];
      if (c.ndrystp < 0 && c.isbal > 0) X.qdwaste[d] = 0.;
      X.wasted[d] = 0;
    }
    X.fuhdye[d] = fuh;
    X.fvhdxe[d] = fvh;
    if (COPY) {
      X.uhdy1e[d] = uh;
      X.vhdx1e[d] = vh;
      X.h1p[d] = HE[d];
    }
    if (c.isdry > 0) {  // :246-253
      X.sub[d] = S.subo[d];
      X.svb[d] = S.svbo[d];
      X.sbx[d] = S.sbxo[d];
      X.sby[d] = S.sbyo[d];
    }
    X.fp1[d] = fp1;
  }
#undef UE
#undef VE
#undef HE
}

// ---------------------------------------------------------------------------
// CALPUV9C(ISTL_) up to its time-level advance (calpuv9c.f90:154-280): the
// QDWASTE reset, the blended density gradients FPGXE/FPGYE, HUTMP/HVTMP, the
// explicit transports from level n-1 (UHDY1E, P1, TSX1, TBX1), the switch
// reset of wetting and drying, FP1.  No swap precedes it: the buffers hold
// the caller's levels.
template <bool BARO>
__global__ void __launch_bounds__(NT) k_begin3(DevStatic S, DevState X, int ntile) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    if (c.isdry > 0 && c.ndrystp < 0) X.qdwaste[d] = 0.;  // :154-160
    double FPGXE = 0., FPGYE = 0.;
    if (BARO && c.baro) {  // :164-190
      double gx, gy;
      baro_faces(S, X, c, q, X.hp, gx, gy);
      FPGXE = c.rold * X.fpgxe[d] + c.rnew * gx;
      FPGYE = c.rold * X.fpgye[d] + c.rnew * gy;
      X.fpgxe[d] = FPGXE;
      X.fpgye[d] = FPGYE;
    }
    double hut, hvt;  // :192-204
    if (c.istl == 2) {
      hut = 0.5 * (X.hu[d] + X.h1u[d]);
      hvt = 0.5 * (X.hv[d] + X.h1v[d]);
      X.hutmp[d] = hut;
      X.hvtmp[d] = hvt;
    } else {
      hut = X.hu[d];
      hvt = X.hv[d];
    }
    const double sub = X.sub[d], svb = X.svb[d];
    const double P1 = X.p1[d];
    X.fuhdye[d] = fuh_face(S, X, c, d, X.uhdy1e[d], hut, P1, X.p1[q.w], sub, FPGXE,
                           X.tsx1[d], X.tbx1[d]);  // :206-222
    X.fvhdxe[d] = fvh_face(S, X, c, d, X.vhdx1e[d], hvt, P1, X.p1[q.s], svb, FPGYE,
                           X.tsy1[d], X.tby1[d]);
    if (c.isdry > 0) {  // :246-262
      X.iscdry[d] = 0;
      X.sub1[d] = sub;
      X.svb1[d] = svb;
      X.sub[d] = S.subo[d];
      X.svb[d] = S.svbo[d];
      X.sbx[d] = S.sbxo[d];
      X.sby[d] = S.sbyo[d];
      X.oldmask[d] = X.lmaskdry[d];
      X.wasted[d] = 0;
    }
    X.fp1[d] = fp1_cell(S, c, q, P1, X.uhdy1e, X.vhdx1e);  // :268-280
  }
}

// calpuv2c.f90:222-243 (calpuv9c.f90:220-240): the implicit bottom drag with
// vegetation (ISITB >= 1) or the vegetation drag alone (ISVEG > 0) of the
// members that have them, after the explicit transports: RCX, RCY of each
// water cell, and FUHDYE, FVHDXE multiplied by them.  HU, HV, UHE, VHE are
// still the entry values here; HUI(L) is 1./HU(L), as the previous step left
// it (:902-906).  Compiled without FMA contraction, in the reference's
// operand order.
__global__ void __launch_bounds__(NT) k_implicit_drag(DevStatic S, DevState X, int ntile,
                                                     const int *act) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m] || !(c.isitb >= 1 || c.isveg > 0)) continue;
    const int d = tile * TILE + threadIdx.x;
    if (S.kind[d] == LAND) continue;
    const double DELT = c.delt;
    double rx, ry;
    if (c.isitb >= 1) {
      const double U = X.ubot[d], V = X.vbot[d];
      double TMPX = 1.0, TMPY = 1.0;
      if (X.uhe[d] != 0.0) TMPX = U * X.hu[d] / X.uhe[d];
      if (X.vhe[d] != 0.0) TMPY = V * X.hv[d] / X.vhe[d];
      const double HUI = 1. / X.hu[d], HVI = 1. / X.hv[d];
      rx = 1. / (1. + TMPX * c.ritb * DELT * HUI * X.stbx[d] *
                          sqrt(X.vu[d] * X.vu[d] + U * U) +
                 DELT * X.fxvege[d]);
      ry = 1. / (1. + TMPY * c.ritb * DELT * HVI * X.stby[d] *
                          sqrt(X.uv[d] * X.uv[d] + V * V) +
                 DELT * X.fyvege[d]);
    } else {
      rx = 1. / (1. + DELT * X.fxvege[d]);
      ry = 1. / (1. + DELT * X.fyvege[d]);
    }
    X.rcx[d] = rx;
    X.rcy[d] = ry;
    X.fuhdye[d] = X.fuhdye[d] * rx;
    X.fvhdxe[d] = X.fvhdxe[d] * ry;
  }
}
void launch_implicit_drag(const Launch &l, const DevStatic &S, const DevState &X,
                          const int *act) {
  k_implicit_drag<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, act);
  count_launches(1);
}

// CALPUV9C(3), the copies of the time-level advance (calpuv9c.f90:282-311);
// the host has rotated the buffers UHDY2E <- UHDY1E <- UHDYE and
// H2P <- H1P <- HP before it.  NCTBC = 1 halves UHDYE on the way (:289-294).
__global__ void __launch_bounds__(NT) k_advance3(DevStatic S, DevState X, int ntile) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    const int d = tile * TILE + threadIdx.x;
    if (S.kind[d] == LAND) continue;
    if (c.nctbc == 1) {
      X.uhdy1e[d] = 0.5 * X.uhdy1e[d];
      X.vhdx1e[d] = 0.5 * X.vhdx1e[d];
    }
    X.p1[d] = X.p[d];
    X.h1u[d] = X.hu[d];
    X.h1v[d] = X.hv[d];
  }
}

// Start of a sweep: reset the per-member minima, symmetry and re-solve flags.
__global__ void k_sweep_reset(Ctl *ctl, const int *act, int nmember) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < nmember; m += gridDim.x * blockDim.x) {
    if (!act[m]) continue;
    ctl[m].ccmnm_int = 1.e+18;
    ctl[m].ccmnm_bc = 1.e+18;
    ctl[m].asym = 0;
    ctl[m].icordry = 0;
    ctl[m].counter = 0u;
  }
}

// ---------------------------------------------------------------------------
// calpuv2c.f90:306-344 (FP, CS, CW, CE, CN, CC) and the member's minimum of
// CC over its non-open-boundary cells (:360-368; the open-boundary cells' CC
// is replaced by SETOPENBC and enters through k_obc_*).  CC > 0 here.
__global__ void __launch_bounds__(NT) k_assemble(DevStatic S, DevState X, int ntile, Ctl *ctl,
                                                const int *act) {
  __shared__ double sh[32];
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m]) continue;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    const uint8_t kd = S.kind[d];
    double mn = 1.e+18;
    if (kd != LAND) {
      const double cc = assemble_cell(S, X, c, q, X.fp1[d], X.fuhdye[d], X.fuhdye[q.e],
                                      X.fvhdxe[d], X.fvhdxe[q.n]);
      if (kd == WATER) mn = cc;
    }
    mn = block_min(mn, sh);
    if (threadIdx.x == 0 && mn < 1.e+18) atomic_min_nonneg(&ctl[m].ccmnm_int, mn);
  }
}

// ---------------------------------------------------------------------------
// SETOPENBC (setopenbc.f90:22-206) + SETOPENBC2 (setopenbc2.f90:17-46) for one
// boundary cell k.  Returns CC of the cell.
__device__ __forceinline__ double obc_cell(const DevStatic &S, const DevState &X,
                                           const DevObc &B, const StepScalars &c, int k, int mt) {
  const int d = B.slot[k], nb = B.nbr[k], side = B.side[k], ispb = B.ispb[k];
  const double D = c.deltd2, G = c.g, HDRY2 = 0.2 * c.hdry;
  X.cc[d] = c.delti * S.dxyp[d];
  X.cs[d] = 0.;
  X.cw[d] = 0.;
  X.ce[d] = 0.;
  X.cn[d] = 0.;
  if (!X.lopenbcdry[d]) {
    double fp = B.pser ? B.pser[k] : 0.0;
    for (int t = 0; t < mt; ++t) {
      const double TC = c.cosv[t], TS = c.sinv[t];
      fp = fp + B.pcb[k * B.mtmax + t] * TC + B.psb[k * B.mtmax + t] * TS;
    }
    if (ispb == 1 || ispb == 2) {  // radiation
      if (side == 0) {  // W, face at LEC(L)
        const double CET = 0.5 * D * G * S.hruo[nb] * rc_x(X, c, nb) * X.huc[nb];
        const double TMP = D * sqrt(G * X.huc[nb]) * S.dxiu[nb];
        X.cc[d] = CET * (1. + TMP) / TMP;
        X.ce[d] = -CET;
        fp = CET * (2. * fp - sqrt(G * X.huc[nb]) * X.fuhdye[nb] * S.dyiu[nb] / X.huc[nb]) / TMP;
      } else if (side == 1) {  // E, own west face
        const double CWT = 0.5 * D * G * S.hruo[d] * rc_x(X, c, d) * X.huc[d];
        const double TMP = D * sqrt(G * X.huc[d]) * S.dxiu[d];
        X.cc[d] = CWT * (1. + TMP) / TMP;
        X.cw[d] = -CWT;
        fp = CWT * (2. * fp + sqrt(G * X.huc[d]) * X.fuhdye[d] * S.dyiu[d] / X.huc[d]) / TMP;
      } else if (side == 2) {  // S, face at LNC(L)
        const double CNT = 0.5 * D * G * S.hrvo[nb] * rc_y(X, c, nb) * X.hvc[nb];
        const double TMP = D * sqrt(G * X.hvc[nb]) * S.dyiv[nb];
        X.cc[d] = CNT * (1. + TMP) / TMP;
        X.cn[d] = -CNT;
        fp = CNT * (2. * fp - sqrt(G * X.hvc[nb]) * X.fvhdxe[nb] * S.dxiv[nb] / X.hvc[nb]) / TMP;
      } else {  // N, own south face
        const double CST = 0.5 * D * G * S.hrvo[d] * rc_y(X, c, d) * X.hvc[d];
        const double TMP = D * sqrt(G * X.hvc[d]) * S.dyiv[d];
        X.cc[d] = CST * (1. + TMP) / TMP;
        X.cs[d] = -CST;
        fp = CST * (2. * fp + sqrt(G * X.hvc[d]) * X.fvhdxe[d] * S.dxiv[d] / X.hvc[d]) / TMP;
      }
    } else {  // clamped elevation
      const double FP1G = fp / G - HDRY2;
      double CT;
      if (FP1G < S.belv[d] || FP1G < S.belv[nb]) {
        fp = (S.belv[d] + HDRY2) * G;
        CT = 0.;
        X.lopenbcdry[d] = 1;
      } else if (side == 0) {
        CT = 0.5 * D * G * S.hruo[nb] * rc_x(X, c, nb) * X.huc[nb];
      } else if (side == 1) {
        CT = 0.5 * D * G * S.hruo[d] * rc_x(X, c, d) * X.huc[d];
      } else if (side == 2) {
        CT = 0.5 * D * G * S.hrvo[nb] * rc_y(X, c, nb) * X.hvc[nb];
      } else {
        CT = 0.5 * D * G * S.hrvo[d] * rc_y(X, c, d) * X.hvc[d];
      }
      X.fp[nb] = X.fp[nb] + CT * fp;
      fp = c.delti * S.dxyp[d] * fp;
    }
    X.fp[d] = fp;
  }
  return X.cc[d];
}

__device__ __forceinline__ void obc2_cell(const DevState &X, const DevObc &B, int k) {
  if (B.ispb[k] != 0) return;
  const int nb = B.nbr[k];
  switch (B.side[k]) {
    case 0: X.cw[nb] = 0.; break;
    case 1: X.ce[nb] = 0.; break;
    case 2: X.cs[nb] = 0.; break;
    default: X.cn[nb] = 0.; break;
  }
}

// Boundary cells in parallel, one thread each (hazard-free layouts only: no
// two cells share an interior target and no target is a boundary cell, so
// SETOPENBC's and SETOPENBC2's writes to the targets commute).  The minimum
// CC of each member's boundary cells goes to ctl[m].ccmnm_bc (atomic min).
__global__ void __launch_bounds__(NT) k_obc_parallel(DevStatic S, DevState X, DevObc B, Ctl *ctl,
                                                    const int *act) {
  const int k = blockIdx.x * NT + threadIdx.x;
  if (k >= B.n) return;
  const int m = B.member[k];
  if (!act[m]) return;
  const double cc = obc_cell(S, X, B, S.sc[m], k, B.mtide[m]);
  obc2_cell(X, B, k);
  atomic_min_nonneg(&ctl[m].ccmnm_bc, cc);
}

// One thread, the reference's exact loop order (layouts where boundary cells
// share or are each other's interior neighbours).
__global__ void k_obc_serial(DevStatic S, DevState X, DevObc B, Ctl *ctl, const int *act) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < B.n; ++k) {
    const int m = B.member[k];
    if (!act[m]) continue;
    const double cc = obc_cell(S, X, B, S.sc[m], k, B.mtide[m]);
    ctl[m].ccmnm_bc = fmin(ctl[m].ccmnm_bc, cc);
  }
  for (int k = 0; k < B.n; ++k)
    if (act[B.member[k]]) obc2_cell(X, B, k);
}

// calpuv2c.f90:150-157: LOPENBCDRY=.FALSE. on the open-boundary cells (ISDRY>0)
__global__ void k_obc_reset(DevStatic S, DevObc B, DevState X, const int *act) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B.n; k += gridDim.x * blockDim.x)
    if (act[B.member[k]] && S.sc[B.member[k]].isdry > 0) X.lopenbcdry[B.slot[k]] = 0;
}

// ---------------------------------------------------------------------------
// calpuv2c.f90:371-399: scale by the member's minimum diagonal.  CE and CN
// are scaled only when the batch holds a possibly unsymmetric member
// (write_cross); otherwise the CG reads CCE(L) = CCW(LE), CCN(L) = CCS(LN).
__global__ void __launch_bounds__(NT) k_scale(DevStatic S, DevState X, DevSystem Y, int ntile,
                                             Ctl *ctl, const int *act, int write_cross) {
  TILE_LOOP(ntile) {
    const int m = S.tile_member[tile];
    if (!act[m]) continue;
    const double CCMNM = fmin(ctl[m].ccmnm_int, ctl[m].ccmnm_bc);
    const double CCMNMI = 1. / CCMNM;
    const int d = tile * TILE + threadIdx.x;
    if (S.kind[d] == LAND) continue;
    Y.ccs[d] = X.cs[d] * CCMNMI;
    Y.ccw[d] = X.cw[d] * CCMNMI;
    Y.ccc[d] = X.cc[d] * CCMNMI;
    Y.fptmp[d] = X.fp[d] * CCMNMI;
    if (write_cross) {
      Y.cce[d] = X.ce[d] * CCMNMI;
      Y.ccn[d] = X.cn[d] * CCMNMI;
    }
  }
}

// MIXED: the FP32 inner operator Ahat = D A D with D = diag(inv_sqrt_diag(CC))
// (unit diagonal): AS(L) = CS(L)*D(L)*D(LS), AW alike; AE, AN only when the
// operator can be unsymmetric (else AE(L)=AW(LE), AN(L)=AS(LN)).  Ahat does
// not depend on the system's scaling, so a step's MIXED solve uses the
// unscaled assembly directly.
__global__ void __launch_bounds__(NT) k_scale32(DevStatic S, SysView V, DevSystem Y, int ntile,
                                               const int *act, int write_cross) {
  TILE_LOOP(ntile) {
    const int m = S.tile_member[tile];
    if (act && !act[m]) continue;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    // the loads first (the stores below could alias them for the compiler)
    const double cc = V.cc[d], cs = V.cs[d], cw = V.cw[d], ccs = V.cc[q.s], ccw = V.cc[q.w];
    const bool ls = S.kind[q.s] == LAND, lw = S.kind[q.w] == LAND;
    double ce = 0., cn = 0., cce = 1., ccn = 1.;
    bool le = true, ln = true;
    if (write_cross) {
      ce = V.ce[d];
      cn = V.cn[d];
      cce = V.cc[q.e];
      ccn = V.cc[q.n];
      le = S.kind[q.e] == LAND;
      ln = S.kind[q.n] == LAND;
    }
    const double di = inv_sqrt_diag(cc);
    auto off = [&](double cnb, bool land, double cx) {
      return land ? 0.f : float(cnb * di * inv_sqrt_diag(cx));
    };
    Y.as32[d] = off(cs, ls, ccs);
    Y.aw32[d] = off(cw, lw, ccw);
    if (write_cross) {
      Y.ae32[d] = off(ce, le, cce);
      Y.an32[d] = off(cn, ln, ccn);
    }
  }
}

// Symmetry of the assembled operator.  The interior assembly gives CE(L) =
// CW(LE) and CN(L) = CS(LN) bit for bit (both are built from the same face's
// values in the same order), so only SETOPENBC/SETOPENBC2 can break it, at an
// open-boundary cell's four faces.  One thread per boundary cell compares
// both coefficients of each face with a water neighbour and flags the member:
// bit 1 (the CG kernels use the four-array form) when the batch's cross
// coefficients are formed, else bit 2, which the host reports as an error.
__global__ void k_obc_asym(DevStatic S, DevState X, DevObc B, Ctl *ctl, const int *act,
                           int write_cross) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B.n; k += gridDim.x * blockDim.x) {
    const int m = B.member[k];
    if (!act[m]) continue;
    const int d = B.slot[k];
    const Nb q = neighbours_of_slot(S.tnbr, d);
    bool a = false;
    if (S.kind[q.e] != LAND) a |= X.ce[d] != X.cw[q.e];
    if (S.kind[q.w] != LAND) a |= X.cw[d] != X.ce[q.w];
    if (S.kind[q.n] != LAND) a |= X.cn[d] != X.cs[q.n];
    if (S.kind[q.s] != LAND) a |= X.cs[d] != X.cn[q.s];
    if (a) atomicOr(&ctl[m].asym, write_cross ? 1 : 2);
  }
}

// ---------------------------------------------------------------------------
// Start of a solve: members not in this sweep are finished from the start.
__global__ void k_solve_reset(Ctl *ctl, Glob *glob, const int *act, int nmember) {
  __shared__ int ninact;
  if (threadIdx.x == 0) ninact = 0;
  __syncthreads();
  for (int m = threadIdx.x; m < nmember; m += blockDim.x) {
    Ctl &k = ctl[m];
    k.done = act[m] ? 0 : 1;
    if (!act[m]) atomicAdd(&ninact, 1);
    k.idone = 0;
    k.iter = 0;
    k.inner_iter = 0;
    k.outer = 0;
    k.status = 0;
    k.parity = 0;
    k.beta = 0.0;
    k.counter = 0u;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    glob->ndone = ninact;
    glob->nidone = 0;
  }
}

// MIXED: start of an outer pass
__global__ void k_outer_reset(Glob *glob) { glob->nidone = 0; }

// CONGRAD in FP64 (congrad.f90:54-187).  Vectors: P (the state array), r,
// p double-buffered (pa/pb, selected by ctl[m].parity), Ap.  z = CCCI*r with
// CCCI = 1./CCC is recomputed where needed instead of stored.

// :54-88 initial residual, z0 = CCCI*r, RPCG.
template <bool MA, bool FOLD>
__global__ void __launch_bounds__(NT) k_cg_init(DevStatic S, DevSystem Y, double *P, Ctl *ctl,
                                               double *part, RedArgs ra) {
  struct A {
    bool skip, asym;
  };
  quad_sweep<1>(
      S, part, [&](int m) { return A{ctl[m].done != 0, unsym<MA>(ctl[m])}; },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        const V4<double> r = residual_row(g, S.kind, P, Y, a.asym);
        const V4<double> c = ld4(Y.ccc + g.d0);
        const V4<double> z = {r.x * rcpT(c.x), r.y * rcpT(c.y), r.z * rcpT(c.z),
                              r.w * rcpT(c.w)};
        if (valid) {
          st4(Y.r + g.d0, r);
          st4(Y.pa + g.d0, z);
          st4(Y.z + g.d0, z);
          v[0] = r.x * z.x + r.y * z.y + r.z * z.z + r.w * z.w;
        }
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0) cg_init_epi(ctl[m], ra.glob, sum[0]);
      }));
}
__global__ void __launch_bounds__(NT) k_red_cg_init(DevStatic S, Ctl *ctl, Glob *glob,
                                                   const double *part) {
  member_reduce<1>(
      S, part, [&](int m) { return ctl[m].done != 0; },
      [&](int m, const double *sum) {
        if (threadIdx.x == 0) cg_init_epi(ctl[m], glob, sum[0]);
      });
}

// :93-125 (p update from the previous iteration, A*p, p.Ap, ALPHA), and the
// previous iteration's X = X + ALPHA*PCG (:133), which needs no other load
// here than X itself (p_old is that PCG, ALPHA still the previous one).
template <bool MA, bool FOLD>
__global__ void __launch_bounds__(NT, MA ? 2 : 3) k_cg_matvec(DevStatic S, DevSystem Y, double *P,
                                                    Ctl *ctl, double *part) {
  struct A {
    bool skip, asym, dox;
    double beta, alpha;
    const double *pold;
    double *pnew;
  };
  quad_sweep<1>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        return A{k.done != 0, unsym<MA>(k), k.iter > 0, k.beta, k.alpha, par ? Y.pb : Y.pa,
                 par ? Y.pa : Y.pb};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        v[0] = matvec_row_z(g, valid, Y.z, Y.ccc, a.pold, a.pnew, Y.ccs, Y.ccw, Y.cce, Y.ccn,
                            Y.ap, a.beta, a.asym, P, a.alpha, a.dox);
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0) cg_matvec_epi(ctl[m], sum[0]);
      }));
}
__global__ void __launch_bounds__(NT) k_red_cg_matvec(DevStatic S, Ctl *ctl, const double *part) {
  member_reduce<1>(
      S, part, [&](int m) { return ctl[m].done != 0; },
      [&](int m, const double *sum) {
        if (threadIdx.x == 0) cg_matvec_epi(ctl[m], sum[0]);
      });
}

// :134-149 (RCG update, RPCGN, RSQ, BETA) and the stop test :165; the P
// update of :133 is the next matrix-vector kernel's (or k_cg_finish's).  With
// no_stop the iteration continues past RSQM and ITERM (kernel timing only).
template <bool FOLD>
__global__ void __launch_bounds__(NT, 5) k_cg_update(DevStatic S, DevSystem Y, Ctl *ctl,
                                                    double *part, RedArgs ra) {
  struct A {
    bool skip;
    double alpha;
  };
  quad_sweep<2>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        return A{k.done != 0, k.alpha};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        update_row<double>(g, valid, nullptr, nullptr, Y.r, Y.ap, Y.ccc, a.alpha, v[0], v[1],
                           Y.z);
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0) cg_update_epi(ctl[m], ra.glob, S.sc[m], sum[0], sum[1], ra.no_stop);
      }));
}
__global__ void __launch_bounds__(NT) k_red_cg_update(DevStatic S, Ctl *ctl, Glob *glob,
                                                     const double *part, int no_stop) {
  member_reduce<2>(
      S, part, [&](int m) { return ctl[m].done != 0; },
      [&](int m, const double *sum) {
        if (threadIdx.x == 0) cg_update_epi(ctl[m], glob, S.sc[m], sum[0], sum[1], no_stop);
      });
}

// After the CG loop: the last iteration's X = X + ALPHA*PCG (congrad.f90:133)
// of every member that iterated, which no further matrix-vector kernel adds.
__global__ void __launch_bounds__(NT) k_cg_finish(DevStatic S, DevSystem Y, double *P,
                                                 const Ctl *ctl) {
  quad_apply(
      S, [&](int m) { return ctl[m].iter == 0; },
      [&](int m, const RowGeo &g) {
        const Ctl &k = ctl[m];
        const double alpha = k.alpha;
        V4<double> x = ld4(P + g.d0);
        const V4<double> p = ld4((k.parity ? Y.pa : Y.pb) + g.d0);
        x.x = x.x + alpha * p.x;
        x.y = x.y + alpha * p.y;
        x.z = x.z + alpha * p.z;
        x.w = x.w + alpha * p.w;
        st4(P + g.d0, x);
      });
}

// ---------------------------------------------------------------------------
// CONGRAD of small members, the whole solve in one CTA per member: the
// member's CG vectors (P, r, z, p double-buffered, Ap) stay in shared memory
// from the first residual to the stop test, its units run SMALL_UNITS at a
// time, and the coefficient arrays are read from global memory.  The rows
// (the same row functions), the per-unit partial sums (warp sums added in
// warp order), the member sums (reduce_partials of a 256-thread CTA) and the
// epilogues are those of k_cg_init, k_cg_matvec, k_cg_update and their member
// reductions, so the iterates equal theirs bit for bit; one launch replaces
// 2 + 4 per iteration.  The rows of a unit past the member's last tile work
// on the member's ghost tile with stores off, so that every access stays in
// the member's window of slots, [its ghost tile, its last tile].
constexpr int SMALL_UNITS = 2;
constexpr int SMALL_NT = SMALL_UNITS * NT;
constexpr int SMALL_CACHED = 2;  // passes whose geometry a thread keeps in registers

// reduce_partials of a 256-thread CTA, by a CTA of SMALL_NT threads (the
// threads past the first 256 add nothing, as block_sum's last stage reads 8
// warps), from the partials in shared memory
constexpr int SMALL_MAX_UNITS = 64;
__device__ __forceinline__ double reduce_partials_256(const double *part, int nblk, double *sh) {
  double s = 0.0;
  for (int base = 0; base < nblk; base += 8 * NT) {
    double v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int i = base + j * NT + int(threadIdx.x);
      v[j] = (threadIdx.x < NT && i < nblk) ? part[i] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) s += v[j];
  }
  return block_sum(s, sh);
}

template <bool MA, int NP>
__global__ void __launch_bounds__(SMALL_NT) k_cg_small(DevStatic S, DevSystem Y, double *P,
                                                      Ctl *ctl, Glob *glob, double *part) {
  extern __shared__ double smv[];
  __shared__ double sh[32];
  __shared__ double wp[2][SMALL_NT / 32];
  __shared__ double qp[2][SMALL_MAX_UNITS];  // the member's per-unit partials
  __shared__ double s_beta, s_alpha;          // the member's control values, as thread 0
  __shared__ int s_done, s_parity;            // leaves them in ctl[m]
  const int m = blockIdx.x;
  if (ctl[m].done) return;  // not in this sweep
  // thread 0 runs the epilogues on ctl[m] and shares what the loop reads
  auto share = [&] {
    if (threadIdx.x == 0) {
      const Ctl &k = ctl[m];
      s_done = k.done;
      s_parity = k.parity;
      s_beta = k.beta;
      s_alpha = k.alpha;
    }
    __syncthreads();
  };
  const int q0 = S.qstart[m], q1 = S.qstart[m + 1], nq = q1 - q0;
  const int ghost = S.quads[q0].y - 1;  // the member's ghost tile, before its tiles
  const int base = ghost * TILE, nsl = (S.tend[m] - ghost) * TILE;
  double *gv[6] = {P, Y.r, Y.z, Y.pa, Y.pb, Y.ap};
  for (int i = threadIdx.x; i < nsl; i += SMALL_NT)
#pragma unroll
    for (int k = 0; k < 6; ++k) smv[k * nsl + i] = gv[k][base + i];
  __syncthreads();
  // pointers that take the slot d of the window to shared memory
  double *const Ps = smv - base;
  DevSystem Ys = Y;
  Ys.r = smv + nsl - base;
  Ys.z = smv + 2 * nsl - base;
  Ys.pa = smv + 3 * nsl - base;
  Ys.pb = smv + 4 * nsl - base;
  Ys.ap = smv + 5 * nsl - base;
  const int qi = threadIdx.x / NT, tq = threadIdx.x % NT;
  const int sub = tq / TPT, q = tq % TPT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool asym = unsym<MA>(ctl[m]);

  // where a thread's rows are in pass p (units u0 + qi, u0 = q0 + p*SMALL_UNITS)
  struct Pass {
    RowGeo g;
    bool have, valid;
  };
  auto pass_of = [&](int u0) {
    const int qd = u0 + qi;
    const bool have = qd < q1;
    const int4 cur = have ? S.quads[qd] : int4{m, ghost, 0, 0};
    const bool valid = have && sub < cur.z;
    const int ti = valid ? cur.y + sub : ghost;
    return Pass{row_geo_nb(__ldg(&S.tnbr[ti]), ti, q), have, valid};
  };
  // NP > 0: the member has at most NP passes, whose geometry is formed once
  // here and kept in registers (the loop then has no dependent loads of the
  // unit table and the tile neighbours)
  Pass pc[NP > 0 ? NP : 1];
  if constexpr (NP > 0) {
#pragma unroll
    for (int p = 0; p < NP; ++p) pc[p] = pass_of(q0 + p * SMALL_UNITS);
  }

  // one sweep of a row body over the member's units, as quad_sweep makes it
  auto sweep = [&](auto body, auto ns_tag) {
    constexpr int NS = decltype(ns_tag)::value;
    auto unit = [&](int u0, const Pass &ps) {
      const int qd = u0 + qi;
      double v[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) v[s] = 0.0;
      body(ps.g, ps.valid, v);
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double x = warp_sum(v[s]);
        if (lane == 0) wp[s][warp] = x;
      }
      __syncthreads();
      if (tq == 0 && ps.have) {
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          double a = 0.0;
#pragma unroll
          for (int w = 0; w < NWARP; ++w) a += wp[s][qi * NWARP + w];
          qp[s][qd - q0] = a;
        }
      }
      __syncthreads();
    };
    if constexpr (NP > 0) {
#pragma unroll
      for (int p = 0; p < NP; ++p)
        if (q0 + p * SMALL_UNITS < q1) unit(q0 + p * SMALL_UNITS, pc[p]);  // CTA-uniform
    } else {
      for (int u0 = q0; u0 < q1; u0 += SMALL_UNITS) unit(u0, pass_of(u0));
    }
  };
  using One = std::integral_constant<int, 1>;
  using Two = std::integral_constant<int, 2>;

  // :54-88
  sweep(
      [&](const RowGeo &g, bool valid, double *v) {
        const V4<double> r = residual_row(g, S.kind, Ps, Ys, asym);
        const V4<double> c = ld4(Y.ccc + g.d0);
        const V4<double> z = {r.x * rcpT(c.x), r.y * rcpT(c.y), r.z * rcpT(c.z),
                              r.w * rcpT(c.w)};
        if (valid) {
          st4(Ys.r + g.d0, r);
          st4(Ys.pa + g.d0, z);
          st4(Ys.z + g.d0, z);
          v[0] = r.x * z.x + r.y * z.y + r.z * z.z + r.w * z.w;
        }
      },
      One{});
  {
    const double rpcg = reduce_partials_256(qp[0], nq, sh);
    if (threadIdx.x == 0) cg_init_epi(ctl[m], glob, rpcg);
    share();
  }
  // :91-169, ITERM bounds the loop (cg_update_epi sets done)
  while (!s_done) {
    {
      const bool par = s_parity;
      const double beta = s_beta;
      const double *pold = par ? Ys.pb : Ys.pa;
      double *pnew = par ? Ys.pa : Ys.pb;
      sweep(
          [&](const RowGeo &g, bool valid, double *v) {
            v[0] = matvec_row_z(g, valid, Ys.z, Y.ccc, pold, pnew, Y.ccs, Y.ccw, Y.cce, Y.ccn,
                                Ys.ap, beta, asym);
          },
          One{});
      const double pap = reduce_partials_256(qp[0], nq, sh);
      if (threadIdx.x == 0) cg_matvec_epi(ctl[m], pap);
      share();
    }
    {
      const double alpha = s_alpha;
      const double *pnew = s_parity ? Ys.pa : Ys.pb;
      sweep(
          [&](const RowGeo &g, bool valid, double *v) {
            update_row<double>(g, valid, Ps, pnew, Ys.r, Ys.ap, Y.ccc, alpha, v[0], v[1], Ys.z);
          },
          Two{});
      const double rz = reduce_partials_256(qp[0], nq, sh);
      const double rr = reduce_partials_256(qp[1], nq, sh);
      if (threadIdx.x == 0) cg_update_epi(ctl[m], glob, S.sc[m], rz, rr, 0);
      share();
    }
  }
  for (int i = threadIdx.x; i < nsl; i += SMALL_NT)
#pragma unroll
    for (int k = 0; k < 6; ++k) gv[k][base + i] = smv[k * nsl + i];
}

// ---------------------------------------------------------------------------
// MIXED outer step: r = b - A*P in FP64 (the FP64 refinement residual), RSQ
// in FP64, and the FP32 scaled inner system's rhs rhat = D^-1/2 r with
// x = 0 and p0 = rhat (k_mx_zinit then forms z0 = M^-1 rhat and p_old = 0 for
// the polynomial members).  rsqm_fac scales the member's RSQM (the MIXED stop,
// below RSQM).  EAGER: the row's loads issued first (kernel variant 3).
// The member's epilogue of the refinement residual: RSQ (of the scaled system,
// as CONGRAD measures it), the stop test on the FP64 RSQ, and the inner
// solve's target.
__device__ __forceinline__ void mx_resid_epi(Ctl &k, const StepScalars &c, const RedArgs &ra,
                                             double rsq, double rz) {
  if (ra.unscaled) {
    const double ccmnm = fmin(k.ccmnm_int, k.ccmnm_bc);
    rsq = rsq / (ccmnm * ccmnm);
  }
  const double rsqm = c.rsqm * ra.rsqm_fac;
  k.rsq64 = rsq;
  k.rsq = rsq;
  k.rpcg = rz;
  k.beta = 0.0;
  k.parity = 0;
  k.inner_iter = 0;
  k.idone = 0;
  k.outer += 1;
  // inner stop on the scaled residual: reduce it by the factor the FP64
  // residual needs to reach 0.1*RSQM, and by at least rel_tol (in norm)
  const double need = (rsq > 0.0) ? ra.margin * 0.1 * rsqm / rsq : 1.0;
  k.rsq_target = rz * fmax(fmin(need, 1.0), ra.rel_tol * ra.rel_tol);
  int fin = 0;
  if (!isfinite(rsq)) {
    k.status = EFDC_XM_NONFINITE;
    fin = 1;
  } else if (!ra.no_stop && (rsq <= rsqm || rz == 0.0)) {
    fin = 1;
  } else if (!ra.no_stop && k.iter >= 2 * c.iterm + 50) {
    k.status = EFDC_XM_CG_MAXITER;  // inner iterations of all passes exhausted
    fin = 1;
  }
  if (fin) {
    k.done = 1;
    atomicAdd(&ra.glob->ndone, 1);
  }
}

template <bool MA, bool EAGER, bool FOLD>
__global__ void __launch_bounds__(NT) k_mx_resid(DevStatic S, SysView V, DevSystem Y,
                                                const double *P, Ctl *ctl, double *part,
                                                RedArgs ra) {
  struct A {
    bool skip, asym;
  };
  quad_sweep<2>(
      S, part, [&](int m) { return A{ctl[m].done != 0, unsym<MA>(ctl[m])}; },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        V4<double> r;
        if constexpr (EAGER)
          r = residual_row_eager(g, S.kind, P, V, a.asym);
        else
          r = residual_row(g, S.kind, P, V, a.asym);
        const V4<double> c = ld4(V.cc + g.d0);
        const V4<float> r32 = {float(r.x * inv_sqrt_diag(c.x)), float(r.y * inv_sqrt_diag(c.y)),
                               float(r.z * inv_sqrt_diag(c.z)), float(r.w * inv_sqrt_diag(c.w))};
        if (valid) {
          st4(Y.r32 + g.d0, r32);
          st4(Y.pa32 + g.d0, r32);
          st4(Y.x32 + g.d0, V4<float>{0.f, 0.f, 0.f, 0.f});
          v[0] = r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w;
          v[1] = double(r32.x) * double(r32.x) + double(r32.y) * double(r32.y) +
                 double(r32.z) * double(r32.z) + double(r32.w) * double(r32.w);
        }
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0) mx_resid_epi(ctl[m], S.sc[m], ra, sum[0], sum[1]);
      }));
}
__global__ void __launch_bounds__(NT) k_red_mx_resid(DevStatic S, Ctl *ctl, const double *part,
                                                    RedArgs ra) {
  member_reduce<2>(
      S, part, [&](int m) { return ctl[m].done != 0; },
      [&](int m, const double *sum) {
        if (threadIdx.x == 0) mx_resid_epi(ctl[m], S.sc[m], ra, sum[0], sum[1]);
      });
}

// MIXED: P += D^-1/2 x32 (the FP32 correction of the scaled system) for the
// members whose inner solve finished.
__global__ void __launch_bounds__(NT) k_mx_apply(DevStatic S, SysView V, DevSystem Y, double *P,
                                                const Ctl *ctl) {
  quad_apply(
      S, [&](int m) { return ctl[m].done || !ctl[m].idone; },
      [&](int m, const RowGeo &g) {
        const Ctl &k = ctl[m];
        V4<double> x = ld4(P + g.d0);
        const V4<double> c = ld4(V.cc + g.d0);
        // the inner solution with its last iteration's alpha*p (which the
        // matrix-vector pass of a next iteration would have added)
        V4<float> d = ld4(Y.x32 + g.d0);
        if (k.inner_iter > 0)
          d = x_plus_alpha_p(d, float(k.alpha), ld4((k.parity ? Y.pa32 : Y.pb32) + g.d0));
        x.x = x.x + double(d.x) * inv_sqrt_diag(c.x);
        x.y = x.y + double(d.y) * inv_sqrt_diag(c.y);
        x.z = x.z + double(d.z) * inv_sqrt_diag(c.z);
        x.w = x.w + double(d.w) * inv_sqrt_diag(c.w);
        st4(P + g.d0, x);
      });
}

// ---------------------------------------------------------------------------
// Standalone CONGRAD: a caller-assembled scaled system (one member).  Land
// slots are made inert (CCC=1, couplings 0, b=0), and the symmetry of the
// given CCE/CCN against CCW(LE)/CCS(LN) is recorded.
__global__ void __launch_bounds__(NT) k_sys_prepare(DevStatic S, DevSystem Y, int ntile, Ctl *ctl) {
  bool asym = false;
  TILE_LOOP(ntile) {
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) {
      Y.ccc[d] = 1.0;
      Y.ccs[d] = Y.ccw[d] = Y.cce[d] = Y.ccn[d] = Y.fptmp[d] = 0.0;
      continue;
    }
    const double cce = Y.cce[d], ccn = Y.ccn[d];
    // a land neighbour is zeroed by this kernel too: compare with 0 there
    const double ccw_e = (S.kind[q.e] == LAND) ? 0.0 : Y.ccw[q.e];
    const double ccs_n = (S.kind[q.n] == LAND) ? 0.0 : Y.ccs[q.n];
    asym |= (cce != ccw_e) || (ccn != ccs_n);
  }
  if (__syncthreads_or(asym) && threadIdx.x == 0) atomicOr(&ctl[0].asym, 1);
}

// ---------------------------------------------------------------------------
// calpuv2c.f90:416-437 face discharges and unit-width discharges.
__global__ void __launch_bounds__(NT) k_backsub(DevStatic S, DevState X, int ntile,
                                               const int *act) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m]) continue;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    // the loads first (the stores below could alias them for the compiler)
    const double P = X.p[d], PW = X.p[q.w], PS = X.p[q.s];
    const double sub = X.sub[d], svb = X.svb[d], fuh = X.fuhdye[d], fvh = X.fvhdxe[d];
    const double hruo = S.hruo[d], hrvo = S.hrvo[d], huc = X.huc[d], hvc = X.hvc[d];
    const double rx = rc_x(X, c, d), ry = rc_y(X, c, d), dyiu = S.dyiu[d], dxiv = S.dxiv[d];
    const double u = sub * (fuh - c.deltd2 * hruo * rx * huc * (P - PW));
    const double v = svb * (fvh - c.deltd2 * hrvo * ry * hvc * (P - PS));
    X.uhdye[d] = u;
    X.vhdxe[d] = v;
    X.uhe[d] = u * dyiu;
    X.vhe[d] = v * dxiv;
  }
}

// calpuv2c.f90:466-486 continuity from H1P, UHDY1E, VHDX1E; CALPUV9C's
// (calpuv9c.f90:500-525) is written DELT*(Q - S/2), from H2P, UHDY2E, VHDX2E
// for ISTL_ = 3 (the views hb, ub, vb).
__global__ void __launch_bounds__(NT) k_continuity(DevStatic S, DevState X, int ntile,
                                                  const int *act) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m]) continue;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    const double *U = X.ub, *V = X.vb;
    if (c.istl == 0)
      X.hp[d] = X.hb[d] + c.deltd2 * S.dxyip[d] *
                              (2. * X.qsume[d] - (X.uhdye[q.e] + U[q.e] - X.uhdye[d] - U[d] +
                                                  X.vhdxe[q.n] + V[q.n] - X.vhdxe[d] - V[d]));
    else
      X.hp[d] = X.hb[d] + c.delt * S.dxyip[d] *
                              (X.qsume[d] - 0.5 * (X.uhdye[q.e] + U[q.e] - X.uhdye[d] - U[d] +
                                                   X.vhdxe[q.n] + V[q.n] - X.vhdxe[d] - V[d]));
  }
}

// calpuv2c.f90:489-535 depths of the open-boundary cells (+ drying of a
// boundary cell).  Concurrent zero-writes to shared faces are benign.
__global__ void k_obc_hp(DevStatic S, DevState X, DevObc B, const int *act) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B.n; k += gridDim.x * blockDim.x) {
    const int m = B.member[k];
    if (!act[m]) continue;
    const StepScalars &c = S.sc[m];
    const int d = B.slot[k];
    double hp = c.gi * X.p[d] - S.belv[d];
    if (c.isdry > 0) {
      const double h1p = X.h1p[d];
      const int obd = X.lopenbcdry[d];
      if ((obd || (h1p < 0.9 * c.hdry && hp < h1p) || hp < 0.) && X.iscdry[d] == 0) {
        if (hp <= 0. && obd)
          hp = 0.2 * c.hdry;
        else
          hp = fmin(fmax(h1p, 0.1 * c.hdry), 0.9 * c.hdry);
        X.iscdry[d] = 1;
        const Nb q = neighbours_of_slot(S.tnbr, d);
        X.sub[d] = 0.;
        X.svb[d] = 0.;
        X.sub[q.e] = 0.;
        X.svb[q.n] = 0.;
        X.sbx[d] = 0.;
        X.sby[d] = 0.;
        X.sbx[q.e] = 0.;
        X.sby[q.n] = 0.;
        X.uhdye[d] = 0.;
        X.uhdye[q.e] = 0.;
        X.vhdxe[d] = 0.;
        X.vhdxe[q.n] = 0.;
        X.lopenbcdry[d] = 1;
        X.cc[d] = c.delti * S.dxyp[d];
        const double p = (hp + S.belv[d]) * c.g;
        X.p[d] = p;
        X.fp1[d] = c.delti * S.dxyp[d] * p;
      }
    }
    X.hp[d] = hp;
  }
}

// ---------------------------------------------------------------------------
// ISDRY>0 and /= 99: P = G*(HP+BELV) (:560-570) fused with the legacy drying
// check of ISDRY 1..97 (:574-603).  All face writes are zeros, so the order
// of the reference's serial loop does not matter.
__global__ void __launch_bounds__(NT) k_wd_legacy(DevStatic S, DevState X, int ntile, Ctl *ctl,
                                                 const int *act) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m] || c.isdry <= 0 || c.isdry == 99) continue;
    const bool check = c.isdry < 98;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    bool flag = false;
    if (S.kind[d] != LAND) {
      const double hp = X.hp[d];
      X.p[d] = c.g * (hp + S.belv[d]);
      bool dry = hp <= c.hdry;
      if (c.istl != 0) {  // calpuv9c.f90:628-662: below HDRY and not rising fast (HPPMC)
        const double HPPMC = X.hb[d];
        dry = hp < c.hdry && (hp < 0.9 * c.hdry || HPPMC < c.hdry) && hp < (HPPMC + 0.1 * c.hdry);
      }
      if (check && dry) {
        if (X.iscdry[d] == 0) {
          X.iscdry[d] = 1;
          flag = true;
        }
        X.sub[d] = 0.;
        X.svb[d] = 0.;
        X.sub[q.e] = 0.;
        X.svb[q.n] = 0.;
        X.sbx[d] = 0.;
        X.sby[d] = 0.;
        X.sbx[q.e] = 0.;
        X.sby[q.n] = 0.;
      }
    }
    if (__syncthreads_or(flag) && threadIdx.x == 0) atomicOr(&ctl[m].icordry, 1);
  }
}

// ISDRY=99 (:606-734), pass 1: P update and each cell's decision, from
// unmodified data.  Code bits: 1 the cell writes its faces; 2 rising fast
// enough to re-wet (then 4/8/16/32 re-open W/E/S/N); 64 the ISCDRY-only
// branches (rising too slowly, or drying).
enum : int { WD_ACT = 1, WD_FAST = 2, WD_RW = 4, WD_RE = 8, WD_RS = 16, WD_RN = 32, WD_SLOW = 64 };

__global__ void __launch_bounds__(NT) k_wd99_decide(DevStatic S, DevState X, int ntile,
                                                   const int *act) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m] || c.isdry != 99) continue;
    const double HDRY = c.hdry, HDRY2 = 2. * HDRY, HDRY90 = 0.9 * HDRY;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) {
      X.wd_act[d] = 0;
      continue;
    }
    const double hp = X.hp[d], h1p = X.hb[d];  // HPPMC: H1P, or H2P in CALPUV9C(3)
    X.p[d] = c.g * (hp + S.belv[d]);
    int a = 0;
    if (hp <= HDRY) {
      const double DHPDT = hp - h1p;
      if (DHPDT > 0.0) {
        a = WD_ACT;
        const double DHPDT2 = (HDRY - h1p) * 0.01;
        if (DHPDT > DHPDT2) {
          a |= WD_FAST;
          if (S.subo[d] > 0.5 && X.uhdye[d] > 0.0 && X.hp[q.w] > HDRY2) a |= WD_RW;
          if (S.subo[q.e] > 0.5 && X.uhdye[q.e] < 0.0 && X.hp[q.e] > HDRY2) a |= WD_RE;
          if (S.svbo[d] > 0.5 && X.vhdxe[d] > 0.0 && X.hp[q.s] > HDRY2) a |= WD_RS;
          if (S.svbo[q.n] > 0.5 && X.vhdxe[q.n] < 0.0 && X.hp[q.n] > HDRY2) a |= WD_RN;
        } else {
          a |= WD_SLOW;
        }
      } else if (hp < HDRY90 || h1p < HDRY) {
        a = WD_ACT | WD_SLOW;
      }
    }
    X.wd_act[d] = a;
  }
}

// ISDRY=99 pass 2: the face values the reference's serial L-order loop
// leaves (a face shared by cells L and LW is last written by L), the ISCDRY
// updates and the re-solve flag, into the *_n scratch arrays.
__global__ void __launch_bounds__(NT) k_wd99_apply(DevStatic S, DevState X, int ntile, Ctl *ctl,
                                                  const int *act) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m] || c.isdry != 99) continue;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    bool flag = false;
    if (S.kind[d] != LAND) {
      const int a = X.wd_act[d], aw = X.wd_act[q.w], as = X.wd_act[q.s];
      const double subo = S.subo[d], svbo = S.svbo[d];
      // the west face SUB(L) (owners: L, then LW as its east face)
      double sub, sbx, svb, sby;
      if (a & WD_ACT) {
        const bool o = a & WD_RW;
        sub = o ? subo : 0.0;
        sbx = o ? S.sbxo[d] : 0.0;
      } else if (aw & WD_ACT) {
        const bool o = aw & WD_RE;
        sub = o ? subo : 0.0;
        sbx = o ? S.sbxo[d] : 0.0;
      } else {
        sub = X.sub[d];
        sbx = X.sbx[d];
      }
      if (a & WD_ACT) {
        const bool o = a & WD_RS;
        svb = o ? svbo : 0.0;
        sby = o ? S.sbyo[d] : 0.0;
      } else if (as & WD_ACT) {
        const bool o = as & WD_RN;
        svb = o ? svbo : 0.0;
        sby = o ? S.sbyo[d] : 0.0;
      } else {
        svb = X.svb[d];
        sby = X.sby[d];
      }
      X.sub_n[d] = sub;
      X.sbx_n[d] = sbx;
      X.svb_n[d] = svb;
      X.sby_n[d] = sby;
      if (a & WD_FAST) {
        const double ww = (a & WD_RW) ? subo : 0.0;
        const double we = (a & WD_RE) ? S.subo[q.e] : 0.0;
        const double ws = (a & WD_RS) ? svbo : 0.0;
        const double wn = (a & WD_RN) ? S.svbo[q.n] : 0.0;
        const double RDRY = ww + we + ws + wn;
        X.iscdry[d] = (RDRY < 0.5) ? 1 : 0;
        // values seen by L before its own writes
        const double SUBW = (aw & WD_ACT) ? ((aw & WD_RE) ? subo : 0.0) : X.sub[d];
        const double SUBE = X.sub[q.e];
        const double SVBS = (as & WD_ACT) ? ((as & WD_RN) ? svbo : 0.0) : X.svb[d];
        const double SVBN = X.svb[q.n];
        if (fabs(ww - SUBW) > 0.5 || fabs(we - SUBE) > 0.5 || fabs(ws - SVBS) > 0.5 ||
            fabs(wn - SVBN) > 0.5)
          flag = true;
      } else if (a & WD_SLOW) {
        if (X.iscdry[d] == 0) {
          X.iscdry[d] = 1;
          flag = true;
        }
      }
    }
    if (__syncthreads_or(flag) && threadIdx.x == 0) atomicOr(&ctl[m].icordry, 1);
  }
}

__global__ void __launch_bounds__(NT) k_wd99_commit(DevStatic S, DevState X, int ntile,
                                                   const int *act) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m] || c.isdry != 99) continue;
    const int d = tile * TILE + threadIdx.x;
    if (S.kind[d] == LAND) continue;
    X.sub[d] = X.sub_n[d];
    X.svb[d] = X.svb_n[d];
    X.sbx[d] = X.sbx_n[d];
    X.sby[d] = X.sby_n[d];
  }
}

// ---------------------------------------------------------------------------
// :838-889 volume wasting of isolated wet cells (ISDRY>0, NDRYSTP<0) and the
// later H1P/QDWASTE fix-up of the wasted cells (:1003-1025).
__global__ void __launch_bounds__(NT) k_fin_waste(DevStatic S, DevState X, int ntile, Ctl *ctl,
                                                 const int *act) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m] || c.isdry <= 0 || c.ndrystp >= 0) continue;
    const int NTMP = abs(c.ndrystp);
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    int nw = 0;
    if (S.kind[d] != LAND) {
      const double hp = X.hp[d];
      if (hp >= c.hdry) {
        const double RDRY = X.sub[d] + X.sub[q.e] + X.svb[d] + X.svb[q.n];
        if (RDRY > 0.5) {
          X.natdry[d] = 0;
        } else {
          const int nat = X.natdry[d] + 1;
          X.natdry[d] = nat;
          if (nat > NTMP) {
            const double bl = S.belv[d];
            double RVAL = 0.0;
            if (S.subo[q.e] > 0.5 && S.belv[q.e] < bl) RVAL = RVAL + 1.;
            if (S.subo[d] > 0.5 && S.belv[q.w] < bl) RVAL = RVAL + 1.;
            if (S.svbo[q.n] > 0.5 && S.belv[q.n] < bl) RVAL = RVAL + 1.;
            if (S.svbo[d] > 0.5 && S.belv[q.s] < bl) RVAL = RVAL + 1.;
            if (RVAL > 0. || hp < c.hdry * 2.) {
              const double HOLDTMP = hp;
              const double hnew = 0.90 * c.hdry;
              X.hp[d] = hnew;
              X.h1p[d] = 0.90 * c.hdry;
              X.natdry[d] = 0;
              // CALPUV9C adds to the QDWASTE zeroed at entry (calpuv9c.f90:919) and keeps it
              X.qdwaste[d] = (c.istl != 0) ? X.qdwaste[d] + c.delti * S.dxyp[d] * (HOLDTMP - hnew)
                             : (c.isbal == 0) ? 0.0 : c.delti * S.dxyp[d] * (HOLDTMP - hnew);
              X.vdwaste[d] = X.vdwaste[d] + S.dxyp[d] * (HOLDTMP - hnew);
              X.wasted[d] = 1;
              nw = 1;
            }
          }
        }
      }
    }
    nw = __syncthreads_count(nw);
    if (threadIdx.x == 0 && nw) atomicAdd(&ctl[m].nwasted, nw);
  }
}

// :893-931 final P (ISDRY=0), HU, HV, LMASKDRY; NEGDEP count (the reciprocals
// HPI, HUI, HVI are formed when downloaded: k_reciprocals).
__global__ void __launch_bounds__(NT) k_fin(DevStatic S, DevState X, int ntile, Ctl *ctl,
                                           const int *act) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    if (!act[m]) continue;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    int neg = 0, bad = 0;
    if (S.kind[d] != LAND) {
      // the loads first (the stores below could alias them for the compiler)
      const double hp = X.hp[d], hpw = X.hp[q.w], hps = X.hp[q.s], belv = S.belv[d];
      const double dxyp = S.dxyp[d], dxypw = S.dxyp[q.w], dxyps = S.dxyp[q.s];
      const double fsgzu = S.fsgzu[d], fsgzv = S.fsgzv[d];
      if (c.isdry == 0) X.p[d] = c.g * (hp + belv);
      const double hu = (dxyp * hp + dxypw * hpw) * fsgzu;
      const double hv = (dxyp * hp + dxyps * hps) * fsgzv;
      X.hu[d] = hu;
      X.hv[d] = hv;
      if (c.isdry > 0) {
        int mask = 1;
        if (hp < c.hdry) {
          int IUW = 0, IUE = 0, IVS = 0, IVN = 0;
          if (X.sub1[d] < 0.5 && X.sub[d] < 0.5) IUE = 1;
          if (X.sub1[q.e] < 0.5 && X.sub[q.e] < 0.5) IUW = 1;
          if (X.svb1[d] < 0.5 && X.svb[d] < 0.5) IVS = 1;
          if (X.svb1[q.n] < 0.5 && X.svb[q.n] < 0.5) IVN = 1;
          if (IUW + IUE + IVS + IVN == 4) mask = 0;
        }
        X.lmaskdry[d] = mask;
      }
      neg = (hp <= 0.) ? 1 : 0;
      bad = isfinite(X.p[d]) ? 0 : 1;
    }
    neg = __syncthreads_count(neg);
    bad = __syncthreads_count(bad);
    if (threadIdx.x == 0) {
      if (neg) atomicAdd(&ctl[m].nneg, neg);
      if (bad) atomicAdd(&ctl[m].nnonfinite, bad);
    }
  }
}

// ---------------------------------------------------------------------------
// Host order <-> tile order.  A staging buffer holds every member's host array
// back to back (member m at element offset moff[m], LC = mlc[m] elements).  A
// land slot receives element LC of its member's array (the ghost value);
// gathers write water slots only.  Both cover the slots [d0, d1).
__global__ void k_scatter(const CopyJob *jobs, int njob, const int *lidx, const int *tile_member,
                          const long long *moff, const int *mlc, int d0, int d1) {
  const int j = blockIdx.y;
  if (j >= njob) return;
  const CopyJob J = jobs[j];
  for (int d = d0 + blockIdx.x * blockDim.x + threadIdx.x; d < d1; d += gridDim.x * blockDim.x) {
    const int L = lidx[d];
    if (L < 2 && J.is_int == 3) continue;  // water-only: leave land slots as they are
    const int m = tile_member[d / TILE];
    const long long src = moff[m] + (L >= 2 ? L : mlc[m]) - 1;
    if (J.is_int == 1 || J.is_int == 2)
      static_cast<int *>(J.dev)[d] = (J.is_int == 1)
                                         ? (static_cast<const int *>(J.host_order)[src] != 0 ? 1 : 0)
                                         : static_cast<const int *>(J.host_order)[src];
    else
      static_cast<double *>(J.dev)[d] = static_cast<const double *>(J.host_order)[src];
  }
}

__global__ void k_gather(const CopyJob *jobs, int njob, const int *lidx, const int *tile_member,
                         const long long *moff, int d0, int d1) {
  const int j = blockIdx.y;
  if (j >= njob) return;
  const CopyJob J = jobs[j];
  for (int d = d0 + blockIdx.x * blockDim.x + threadIdx.x; d < d1; d += gridDim.x * blockDim.x) {
    const int L = lidx[d];
    if (L < 2) continue;
    const long long dst = moff[tile_member[d / TILE]] + L - 1;
    if (J.is_int == 1 || J.is_int == 2)
      static_cast<int *>(const_cast<void *>(J.host_order))[dst] = static_cast<const int *>(J.dev)[d];
    else
      static_cast<double *>(const_cast<void *>(J.host_order))[dst] =
          static_cast<const double *>(J.dev)[d];
  }
}

// ---------------------------------------------------------------------------
// launch wrappers
// dst[idx[i]] = val[i]: a member's values into tile order (set-up only).
__global__ void k_put(const int *idx, const double *val, int n, double *dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[idx[i]] = val[i];
}
void launch_put(cudaStream_t st, const int *idx, const double *val, int n, double *dst) {
  if (n <= 0) return;
  k_put<<<std::min((n + 255) / 256, 4096), 256, 0, st>>>(idx, val, n, dst);
  count_launches(1);
}
__global__ void k_put_int(const int *idx, const int *val, int n, int *dst) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[idx[i]] = val[i];
}
void launch_put_int(cudaStream_t st, const int *idx, const int *val, int n, int *dst) {
  if (n <= 0) return;
  k_put_int<<<std::min((n + 255) / 256, 4096), 256, 0, st>>>(idx, val, n, dst);
  count_launches(1);
}

static int blocks_per_sm(const void *kernel);
// The grid of a cell kernel whose resident CTAs per SM differ from the
// others': its own occupancy times the SMs, at most one CTA per tile.
template <class K>
static int cell_grid(const Launch &l, K kernel) {
  const int per_sm = blocks_per_sm(reinterpret_cast<const void *>(kernel));
  return std::max(1, std::min(l.ntile - 1, l.nsm * per_sm));
}
void launch_begin(const Launch &l, const DevStatic &S, const DevState &X, const int *act,
                  bool copy) {
  if (l.baro) {
    k_calebi<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, act);
    count_launches(1);
  }
  if (l.baro && copy)
    k_begin<true, true><<<cell_grid(l, k_begin<true, true>), NT, 0, l.stream>>>(S, X, l.ntile,
                                                                              act);
  else if (l.baro)
    k_begin<true, false><<<cell_grid(l, k_begin<true, false>), NT, 0, l.stream>>>(S, X, l.ntile,
                                                                                act);
  else if (copy)
    k_begin<false, true><<<cell_grid(l, k_begin<false, true>), NT, 0, l.stream>>>(S, X, l.ntile,
                                                                                act);
  else
    k_begin<false, false><<<cell_grid(l, k_begin<false, false>), NT, 0, l.stream>>>(
        S, X, l.ntile, act);
  count_launches(1);
}
void launch_begin3(const Launch &l, const DevStatic &S, const DevState &X, const int *act) {
  if (l.baro) {
    k_calebi<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, act);  // calpuv9c.f90:145
    count_launches(1);
    k_begin3<true><<<cell_grid(l, k_begin3<true>), NT, 0, l.stream>>>(S, X, l.ntile);
  } else {
    k_begin3<false><<<cell_grid(l, k_begin3<false>), NT, 0, l.stream>>>(S, X, l.ntile);
  }
  count_launches(1);
}
void launch_advance3(const Launch &l, const DevStatic &S, const DevState &X) {
  k_advance3<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile);
  count_launches(1);
}
void launch_sweep_reset(const Launch &l, Ctl *ctl, const int *act, int nmember) {
  k_sweep_reset<<<(nmember + 255) / 256, 256, 0, l.stream>>>(ctl, act, nmember);
  count_launches(1);
}
void launch_assemble(const Launch &l, const DevStatic &S, const DevState &X, Ctl *ctl,
                     const int *act) {
  k_assemble<<<cell_grid(l, k_assemble), NT, 0, l.stream>>>(S, X, l.ntile, ctl, act);
  count_launches(1);
}
void launch_obc(const Launch &l, const DevStatic &S, const DevState &X, const DevObc &B, Ctl *ctl,
                const int *act, bool serial, int write_cross) {
  if (B.n == 0) return;
  if (serial)
    k_obc_serial<<<1, 1, 0, l.stream>>>(S, X, B, ctl, act);
  else
    k_obc_parallel<<<(B.n + NT - 1) / NT, NT, 0, l.stream>>>(S, X, B, ctl, act);
  k_obc_asym<<<(B.n + NT - 1) / NT, NT, 0, l.stream>>>(S, X, B, ctl, act, write_cross);
  count_launches(2);
}
void launch_obc_reset(const Launch &l, const DevStatic &S, const DevObc &B, const DevState &X,
                      const int *act) {
  if (B.n == 0) return;
  k_obc_reset<<<(B.n + 255) / 256, 256, 0, l.stream>>>(S, B, X, act);
  count_launches(1);
}
void launch_scale(const Launch &l, const DevStatic &S, const DevState &X, const DevSystem &Y,
                  Ctl *ctl, const int *act, int mixed, int write_cross) {
  if (mixed) {  // the FP32 operator straight from the unscaled assembly
    const SysView V{X.fp, X.cc, X.cs, X.cw, X.ce, X.cn, 1};
    k_scale32<<<l.grid, NT, 0, l.stream>>>(S, V, Y, l.ntile, act, write_cross);
  } else {
    k_scale<<<l.grid, NT, 0, l.stream>>>(S, X, Y, l.ntile, ctl, act, write_cross);
  }
  count_launches(1);
}
void launch_solve_reset(const Launch &l, Ctl *ctl, Glob *glob, const int *act, int nmember) {
  k_solve_reset<<<1, 256, 0, l.stream>>>(ctl, glob, act, nmember);
  count_launches(1);
}
void launch_outer_reset(const Launch &l, Glob *glob) {
  k_outer_reset<<<1, 1, 0, l.stream>>>(glob);
  count_launches(1);
}
// one CTA per member (grid-stride past 1024 members)
static int reduce_grid(const DevStatic &S) { return std::min(S.nmember, 1024); }

// Resident CTAs per SM of a kernel, looked up once per process and kernel.
static int blocks_per_sm(const void *kernel) {
  static std::mutex mu;
  static std::map<const void *, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int a = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, kernel, NT, 0);
  a = a > 0 ? a : 1;
  cache[kernel] = a;
  return a;
}

// One wave of a quad kernel: its own resident CTAs per SM times the SMs, at
// most one CTA per quad.
template <class K>
static int quad_grid(const Launch &l, const DevStatic &S, K kernel) {
  const int per_sm = blocks_per_sm(reinterpret_cast<const void *>(kernel));
  return std::max(1, std::min(S.nquad, l.nsm * per_sm));
}

template <bool F>
static void cg_init_kernel(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P,
                           Ctl *ctl, double *part, const RedArgs &ra) {
  if (l.may_asym)
    k_cg_init<true, F><<<quad_grid(l, S, k_cg_init<true, F>), NT, 0, l.stream>>>(S, Y, P, ctl,
                                                                                part, ra);
  else
    k_cg_init<false, F><<<quad_grid(l, S, k_cg_init<false, F>), NT, 0, l.stream>>>(S, Y, P, ctl,
                                                                                  part, ra);
  count_launches(1);
}
void launch_cg_init(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P, Ctl *ctl,
                    Glob *glob, double *part) {
  RedArgs ra{};
  ra.glob = glob;
  if (l.fold) {
    cg_init_kernel<true>(l, S, Y, P, ctl, part, ra);
    return;
  }
  cg_init_kernel<false>(l, S, Y, P, ctl, part, ra);
  launch_chan_res64(l, S, Y, P, ctl, part);
  k_red_cg_init<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, glob, part);
  count_launches(1);
}
// Shared memory of k_cg_small for windows of up to `slots` slots (its six
// vectors); false when that is more than a CTA can have.
bool cg_small_fits(int slots) {
  return size_t(slots) * 6 * sizeof(double) <= size_t(SMALL_SMEM_MAX) &&
         slots / (TILES_PER_CTA * TILE) <= SMALL_MAX_UNITS;
}
void launch_cg_small(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P,
                     Ctl *ctl, Glob *glob, double *part, int max_slots, int max_units,
                     int nmember) {
  const size_t smem = size_t(max_slots) * 6 * sizeof(double);
  static std::mutex mu;
  static bool set = false;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!set) {
      for (const void *k : {reinterpret_cast<const void *>(k_cg_small<true, 0>),
                            reinterpret_cast<const void *>(k_cg_small<false, 0>),
                            reinterpret_cast<const void *>(k_cg_small<true, SMALL_CACHED>),
                            reinterpret_cast<const void *>(k_cg_small<false, SMALL_CACHED>)})
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SMALL_SMEM_MAX);
      set = true;
    }
  }
  // members of at most SMALL_CACHED passes keep their geometry in registers
  const bool cached = max_units <= SMALL_CACHED * SMALL_UNITS;
  if (l.may_asym && cached)
    k_cg_small<true, SMALL_CACHED><<<nmember, SMALL_NT, smem, l.stream>>>(S, Y, P, ctl, glob,
                                                                         part);
  else if (l.may_asym)
    k_cg_small<true, 0><<<nmember, SMALL_NT, smem, l.stream>>>(S, Y, P, ctl, glob, part);
  else if (cached)
    k_cg_small<false, SMALL_CACHED><<<nmember, SMALL_NT, smem, l.stream>>>(S, Y, P, ctl, glob,
                                                                          part);
  else
    k_cg_small<false, 0><<<nmember, SMALL_NT, smem, l.stream>>>(S, Y, P, ctl, glob, part);
  count_launches(1);
}
template <bool F>
static void cg_matvec_kernel(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P,
                             Ctl *ctl, double *part) {
  if (l.may_asym)
    k_cg_matvec<true, F><<<quad_grid(l, S, k_cg_matvec<true, F>), NT, 0, l.stream>>>(S, Y, P, ctl,
                                                                                    part);
  else
    k_cg_matvec<false, F><<<quad_grid(l, S, k_cg_matvec<false, F>), NT, 0, l.stream>>>(S, Y, P,
                                                                                      ctl, part);
  count_launches(1);
}
void launch_cg_matvec(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P,
                      Ctl *ctl, double *part) {
  if (l.fold) {
    cg_matvec_kernel<true>(l, S, Y, P, ctl, part);
    return;
  }
  cg_matvec_kernel<false>(l, S, Y, P, ctl, part);
  launch_chan_mv64(l, S, Y, ctl, part);
  k_red_cg_matvec<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, part);
  count_launches(1);
}
void launch_cg_update(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      Glob *glob, double *part, int no_stop) {
  RedArgs ra{};
  ra.glob = glob;
  ra.no_stop = no_stop;
  if (l.fold) {
    k_cg_update<true><<<quad_grid(l, S, k_cg_update<true>), NT, 0, l.stream>>>(S, Y, ctl, part,
                                                                              ra);
    count_launches(1);
    return;
  }
  k_cg_update<false><<<quad_grid(l, S, k_cg_update<false>), NT, 0, l.stream>>>(S, Y, ctl, part,
                                                                              ra);
  k_red_cg_update<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, glob, part, no_stop);
  count_launches(2);
}
void launch_cg_finish(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P,
                      const Ctl *ctl) {
  k_cg_finish<<<quad_grid(l, S, k_cg_finish), NT, 0, l.stream>>>(S, Y, P, ctl);
  count_launches(1);
}
void launch_cg_iter(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P, Ctl *ctl,
                    Glob *glob, double *part) {
  launch_cg_matvec(l, S, Y, P, ctl, part);
  launch_cg_update(l, S, Y, ctl, glob, part, 0);
}
template <bool F>
static void mx_resid_kernel(const Launch &l, const DevStatic &S, const SysView &V,
                            const DevSystem &Y, const double *P, Ctl *ctl, double *part,
                            const RedArgs &ra) {
  if (l.variant == 3) {
    if (l.may_asym)
      k_mx_resid<true, true, F><<<quad_grid(l, S, k_mx_resid<true, true, F>), NT, 0,
                                  l.stream>>>(S, V, Y, P, ctl, part, ra);
    else
      k_mx_resid<false, true, F><<<quad_grid(l, S, k_mx_resid<false, true, F>), NT, 0,
                                   l.stream>>>(S, V, Y, P, ctl, part, ra);
  } else if (l.may_asym) {
    k_mx_resid<true, false, F><<<quad_grid(l, S, k_mx_resid<true, false, F>), NT, 0,
                                 l.stream>>>(S, V, Y, P, ctl, part, ra);
  } else {
    k_mx_resid<false, false, F><<<quad_grid(l, S, k_mx_resid<false, false, F>), NT, 0,
                                  l.stream>>>(S, V, Y, P, ctl, part, ra);
  }
  count_launches(1);
}
void launch_mx_resid(const Launch &l, const DevStatic &S, const SysView &V, const DevSystem &Y,
                     const double *P, Ctl *ctl, Glob *glob, double *part, double rsqm_fac,
                     double rel_tol, int no_stop) {
  RedArgs ra{};
  ra.glob = glob;
  ra.rsqm_fac = rsqm_fac;
  ra.rel_tol = rel_tol;
  ra.margin = l.inner_margin;
  ra.no_stop = no_stop;
  ra.unscaled = V.unscaled;
  if (l.fold) {
    mx_resid_kernel<true>(l, S, V, Y, P, ctl, part, ra);
  } else {
    mx_resid_kernel<false>(l, S, V, Y, P, ctl, part, ra);
    launch_chan_resmx(l, S, V, Y, P, ctl, part);
    k_red_mx_resid<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, part, ra);
    count_launches(1);
  }
  launch_mx_zinit(l, S, Y, ctl, part);  // z0 = M^-1 r0 of the inner solve
}
void launch_mx_apply(const Launch &l, const DevStatic &S, const SysView &V, const DevSystem &Y,
                     double *P, const Ctl *ctl) {
  k_mx_apply<<<quad_grid(l, S, k_mx_apply), NT, 0, l.stream>>>(S, V, Y, P, ctl);
  count_launches(1);
}
void launch_backsub(const Launch &l, const DevStatic &S, const DevState &X, const int *act) {
  k_backsub<<<cell_grid(l, k_backsub), NT, 0, l.stream>>>(S, X, l.ntile, act);
  count_launches(1);
  k_continuity<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, act);
  count_launches(1);
}
void launch_obc_hp(const Launch &l, const DevStatic &S, const DevState &X, const DevObc &B,
                   const int *act) {
  if (B.n == 0) return;
  k_obc_hp<<<(B.n + 255) / 256, 256, 0, l.stream>>>(S, X, B, act);
  count_launches(1);
}
void launch_wetdry(const Launch &l, const DevStatic &S, const DevState &X, Ctl *ctl,
                   const int *act, bool any_legacy, bool any99) {
  if (any_legacy) {
    k_wd_legacy<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, ctl, act);
    count_launches(1);
  }
  if (any99) {
    k_wd99_decide<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, act);
    count_launches(1);
    k_wd99_apply<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, ctl, act);
    count_launches(1);
    k_wd99_commit<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, act);
    count_launches(1);
  }
}
void launch_final(const Launch &l, const DevStatic &S, const DevState &X, Ctl *ctl,
                  const int *act, bool any_waste) {
  if (any_waste) {
    k_fin_waste<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, ctl, act);
    count_launches(1);
  }
  k_fin<<<l.grid, NT, 0, l.stream>>>(S, X, l.ntile, ctl, act);
  count_launches(1);
}
// The autotuner's initial guess for timing a solve: P at the entry of the
// last step, which a step without wetting and drying left as G*(HP+BELV)
// (calpuv2c.f90:893-896) and whose HP the time-level advance kept in H1P.
__global__ void __launch_bounds__(NT) k_tune_guess(DevStatic S, DevState X, double *out,
                                                  int ntile) {
  TILE_LOOP(ntile) {
    TILE_MEMBER(S);
    const int d = tile * TILE + threadIdx.x;
    out[d] = (S.kind[d] == LAND) ? X.p[d] : c.g * (X.h1p[d] + S.belv[d]);
  }
}
void launch_tune_guess(const Launch &l, const DevStatic &S, const DevState &X, double *out) {
  k_tune_guess<<<l.grid, NT, 0, l.stream>>>(S, X, out, l.ntile);
  count_launches(1);
}

// HPI, HUI, HVI (calpuv2c.f90:896-906) from the final HP, HU, HV: outputs
// only (nothing on the device reads them), formed when they are downloaded;
// tiles [t0, t1).
__global__ void __launch_bounds__(NT) k_reciprocals(DevStatic S, DevState X, int t0, int t1) {
  for (int tile = t0 + blockIdx.x; tile < t1; tile += gridDim.x) {
    const int d = tile * TILE + threadIdx.x;
    if (S.kind[d] == LAND) continue;
    X.hpi[d] = 1. / X.hp[d];
    X.hui[d] = 1. / X.hu[d];
    X.hvi[d] = 1. / X.hv[d];
  }
}
void launch_reciprocals(const Launch &l, const DevStatic &S, const DevState &X, int t0, int t1) {
  if (t1 <= t0) return;
  k_reciprocals<<<std::min(l.grid, t1 - t0), NT, 0, l.stream>>>(S, X, t0, t1);
  count_launches(1);
}

// ---------------------------------------------------------------------------
// Bottom-stress producer: CALTBXY's drag coefficients (caltbxy.f90:476-539,
// ISWAVE = ISVEG = ISMUD = ISITB = 0: CDLIMIT = 0.5) and the bottom stresses of
// hdmt2t.f90:670-684, over the wet cells (LWET: every cell with ISDRY = 0,
// else the cells with LMASKDRY); the faces of the cells of LDRY (not wet, and
// dry at entry or N < NTSTBC+1) get TBX = TBY = 0 (caltbxy.f90:213-229), the
// others keep theirs.  HU, HV, LMASKDRY and the entry mask are the state the
// last step left on the device.
__global__ void __launch_bounds__(NT) k_tbxy(DevStatic S, DevState X, DevBed Bd,
                                            const DragScalars *ds, int ntile) {
  TILE_LOOP(ntile) {
    const DragScalars &q = ds[S.tile_member[tile]];
    if (!q.on) continue;
    const Nb nb = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = nb.d;
    if (S.kind[d] == LAND) continue;
    if (!(q.isdry == 0 || X.lmaskdry[d] != 0)) {
      auto ldry = [&](int s) {
        return S.kind[s] != LAND && X.lmaskdry[s] == 0 &&
               (X.oldmask[s] != 0 || q.n < q.ntstbc + 1);
      };
      const bool dd = ldry(d);  // TBX(L), TBX(LEC(L)) of the cells L of LDRY
      double *TBX = const_cast<double *>(X.tbx), *TBY = const_cast<double *>(X.tby);
      if (dd || ldry(nb.w)) TBX[d] = 0.;
      if (dd || ldry(nb.s)) TBY[d] = 0.;
      continue;
    }
    const double U = Bd.ub[d], V = Bd.vb[d], VU = Bd.vu[d], UV = Bd.uv[d];
    const double hu = X.hu[d], hv = X.hv[d];
    const double stbxo = Bd.stbxo[d], stbyo = Bd.stbyo[d];
    double stbx, stby;
    if (Bd.zbr[d] <= 1.E-6) {  // :480-502 smooth (viscous) drag
      const double UMAG = sqrt(U * U + VU * VU + 1.E-12);
      const double VMAG = sqrt(UV * UV + V * V + 1.E-12);
      const double CDMAXU = 0.5 * stbxo * hu / (q.delt * UMAG);
      const double CDMAXV = 0.5 * stbyo * hv / (q.delt * VMAG);
      double VISDHU = 0.0, VISDHV = 0.0;
      if (UMAG > 0.0) VISDHU = (q.vismud * (1. / hu) / UMAG) * (2. / 7.);
      if (VMAG > 0.0) VISDHV = (q.vismud * (1. / hv) / VMAG) * (2. / 7.);
      stbx = fmin(CDMAXU, q.visfac * q.avcon * stbxo * VISDHU);
      stby = fmin(CDMAXV, q.visfac * q.avcon * stbyo * VISDHV);
    } else {  // :504-537 rough (log-law) drag
      const double UMAG = sqrt(VU * VU + U * U + 1.E-12);
      const double VMAG = sqrt(UV * UV + V * V + 1.E-12);
      const double CDMAXU = 0.5 * stbxo * hu / (q.delt * UMAG);
      const double CDMAXV = 0.5 * stbyo * hv / (q.delt * VMAG);
      const double zu = Bd.zbratu[d], zv = Bd.zbratv[d];
      const double HURTMP = fmax(zu, Bd.h1u[d]);
      const double HVRTMP = fmax(zv, Bd.h1v[d]);
      if (q.kc1) {
        const double lu = log(fmax(0.5 * HURTMP / zu, 7.5)) - 1.;
        const double lv = log(fmax(0.5 * HVRTMP / zv, 7.5)) - 1.;
        stbx = stbxo * .16 / (lu * lu);
        stby = stbyo * .16 / (lv * lv);
      } else {
        const double lu = log(fmax(1. + Bd.sgzuu[d] * HURTMP / zu, 7.5));
        const double lv = log(fmax(1. + Bd.sgzvv[d] * HVRTMP / zv, 7.5));
        stbx = q.avcon * stbxo * .16 / (lu * lu);
        stby = q.avcon * stbyo * .16 / (lv * lv);
      }
      stbx = fmin(CDMAXU, stbx);
      stby = fmin(CDMAXV, stby);
    }
    Bd.stbx[d] = stbx;
    Bd.stby[d] = stby;
    // hdmt2t.f90:682-683 (TBX, TBY are inputs of the step: written here only)
    const_cast<double *>(X.tbx)[d] = (q.avcon1 * (1. / hu) + stbx * sqrt(VU * VU + U * U)) * U;
    const_cast<double *>(X.tby)[d] = (q.avcon1 * (1. / hv) + stby * sqrt(UV * UV + V * V)) * V;
  }
}
// The bed's derived arrays of member m's slots (caltbxy.f90:81-90, layer 1):
// ZBRATU from the west neighbour's DXP*ZBR (a land neighbour is the ghost
// cell LC, LWC(L) = LC: gu = DXP(LC)*ZBR(LC), gv = DYP(LC)*ZBR(LC) of the
// member), SGZUU = 0.5*MAX(DZC, SGZU).
__global__ void __launch_bounds__(NT) k_bed(DevStatic S, DevBed Bd, const double *dxp,
                                           const double *dyp, const double *dzc1,
                                           const double *sgzu1, const double *sgzv1, double gu,
                                           double gv, int t0, int t1) {
  for (int tile = t0 + blockIdx.x; tile < t1; tile += gridDim.x) {
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    const double *Z = Bd.zbr;
    const double wu = S.kind[q.w] == LAND ? gu : dxp[q.w] * Z[q.w];
    const double wv = S.kind[q.s] == LAND ? gv : dyp[q.s] * Z[q.s];
    const_cast<double *>(Bd.zbratu)[d] = 0.5 * (wu + dxp[d] * Z[d]) * S.dxiu[d];
    const_cast<double *>(Bd.zbratv)[d] = 0.5 * (wv + dyp[d] * Z[d]) * S.dyiv[d];
    const_cast<double *>(Bd.sgzuu)[d] = 0.5 * fmax(dzc1[d], sgzu1[d]);
    const_cast<double *>(Bd.sgzvv)[d] = 0.5 * fmax(dzc1[d], sgzv1[d]);
  }
}
void launch_bed(cudaStream_t st, const DevStatic &S, const DevBed &Bd, const double *dxp,
                const double *dyp, const double *dzc1, const double *sgzu1, const double *sgzv1,
                double gu, double gv, int t0, int t1) {
  if (t1 <= t0) return;
  k_bed<<<std::min(t1 - t0, 4096), NT, 0, st>>>(S, Bd, dxp, dyp, dzc1, sgzu1, sgzv1, gu, gv, t0,
                                                t1);
  count_launches(1);
}

void launch_tbxy(const Launch &l, const DevStatic &S, const DevState &X, const DevBed &Bd,
                 const DragScalars *ds) {
  k_tbxy<<<cell_grid(l, k_tbxy), NT, 0, l.stream>>>(S, X, Bd, ds, l.ntile);
  count_launches(1);
}

// Small control blocks between device memory and mapped pinned host memory,
// copied by a kernel: loads and stores over the link use no copy engine, so
// they do not queue behind bulk copies in flight on other streams.
__global__ void k_words(const unsigned *src, unsigned *dst, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = src ? src[i] : 0u;
}
void launch_words(cudaStream_t st, void *dst, const void *src, size_t bytes) {
  const int n = int(bytes / sizeof(unsigned));
  if (n <= 0) return;
  k_words<<<std::min((n + 255) / 256, 1184), 256, 0, st>>>(static_cast<const unsigned *>(src),
                                                           static_cast<unsigned *>(dst), n);
  count_launches(1);
}

void launch_scatter(cudaStream_t st, const CopyJob *jobs, int njob, const int *lidx,
                    const int *tile_member, const long long *moff, const int *mlc, int d0,
                    int d1) {
  if (njob == 0 || d1 <= d0) return;
  dim3 g(std::min((d1 - d0 + 255) / 256, 2048), njob);
  k_scatter<<<g, 256, 0, st>>>(jobs, njob, lidx, tile_member, moff, mlc, d0, d1);
  count_launches(1);
}
void launch_gather(cudaStream_t st, const CopyJob *jobs, int njob, const int *lidx,
                   const int *tile_member, const long long *moff, int d0, int d1) {
  if (njob == 0 || d1 <= d0) return;
  dim3 g(std::min((d1 - d0 + 255) / 256, 2048), njob);
  k_gather<<<g, 256, 0, st>>>(jobs, njob, lidx, tile_member, moff, d0, d1);
  count_launches(1);
}
void launch_sys_prepare(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                        int mixed) {
  k_sys_prepare<<<l.grid, NT, 0, l.stream>>>(S, Y, l.ntile, ctl);
  count_launches(1);
  if (mixed) {  // the standalone system may be unsymmetric: always the 4-array form
    const SysView V{Y.fptmp, Y.ccc, Y.ccs, Y.ccw, Y.cce, Y.ccn, 0};
    k_scale32<<<l.grid, NT, 0, l.stream>>>(S, V, Y, l.ntile, nullptr, 1);
    count_launches(1);
  }
}

// the CTAs per SM of the grid-stride cell kernels (k_begin and k_assemble hold
// more values and run on grids of their own, cell_grid)
int occupancy_blocks_per_sm() {
  int c = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_fin, NT, 0);
  return c > 0 ? c : 1;
}

int occupancy_blocks_per_sm_cg() {
  int a = 0, b = 0, c = 0, d = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_mx_apply, NT, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_cg_update<false>, NT, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_cg_init<true, false>, NT, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, k_mx_resid<true, false, false>, NT, 0);
  const int m = std::min(std::min(a, b), std::min(c, d));
  return m > 0 ? m : 1;
}

}  // namespace xm
