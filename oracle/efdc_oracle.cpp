// efdc_oracle.cpp -- TEST INFRASTRUCTURE ONLY: CPU FP64 restatement of EFDC+
// 8.5 CALPUV2C / CALPUV9C / CONGRAD / CONGRADC / SUBCHAN / CALEBI (standard sigma) /
// SETOPENBC / SETOPENBC2 / NEGDEP (check part) / CALTBXY (bed drag) / CALEXP2T
// (external-mode terms).
// Parity against the reference is UNPINNED (no compiler, no reference tests);
// see efdc_oracle.h.  Each block cites the Fortran it restates.
//
// Build: g++ -O2 -std=c++17 -fopenmp -ffp-contract=off -fPIC -shared
// (oracle/Makefile).  -ffp-contract=off keeps every a*b+c as two roundings,
// as the SSE2 ReleaseDP64 build does.

#include "efdc_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// 1-based view of a caller array: element L is at b[L-1].
template <class T>
struct F {
  T *b;
  T &operator[](long L) const { return b[L - 1]; }
};

struct Side {
  int n = 0;
  std::vector<int> l, ispb;        // 1..n stored at [ll-1]
  std::vector<double> pcb, psb;    // [(m-1)*n + (ll-1)]
};

// Sub-grid channels (GLOBAL's MDCHH arrays), channel NMD at [NMD-1].
struct Channels {
  int n = 0;
  std::vector<int> typ, lh, lu, lv;
  std::vector<double> len, fric, dxp, dyp;  // dxp/dyp 1-based over 1..LC
  // SUBCHAN's per-step outputs and the step-start copies of CALPUV2C
  std::vector<double> cu, cv, chh, qut, qvt;
  std::vector<int> iact;
};

}  // namespace

struct oracle_ctx {
  int la = 0, lc = 0, nthreads = 1, noptimal = 1, ldmopt = 1;
  // static arrays, 1-based (index 0 unused), length lc+2
  std::vector<int> lnc, lsc, lec, lwc;
  std::vector<double> dxyp, dxyip, dxiu, dyiu, dxiv, dyiv, dxyu, dxyv, hruo,
      hrvo, subo, svbo, sbxo, sbyo, belv;
  int mtide = 0;
  std::vector<double> tcp;
  Side side[4];
  std::vector<int> lobcs;  // S, W, E, N order (setbcs.f90:882-935)
  // SAVEd work arrays of CALPUV2C / CONGRAD
  std::vector<double> fp1, fp, fuhdye, fvhdxe, cs, cw, ce, cn, cc, ccs, ccw,
      cce, ccn, ccc, ccci, fptmp, rcx, rcy, sub1, svb1, fsgzu, fsgzv, uhdy1e,
      vhdx1e;
  std::vector<double> pcg, pnv, pev, pwv, psv, rcg, apcg, tmpcg;
  std::vector<int> oldmask;
  Channels ch;
  std::vector<double> p1;  // P at entry (P1, calpuv2c.f90:259)
  // CALEBI: layers (DZCC, ZZC of the first call, layer k at [k*(lc+2) + L])
  // and the buoyancy integrals, kept between calls like the module arrays
  int kc = 0;
  std::vector<double> dzc, zz, bi1, bi2, be;
  // bottom-stress producer (CALTBXY): the bed, 1-based over 1..LC, and the
  // drag coefficients kept between calls (zero before the first)
  bool bed = false;
  int bed_kc = 0;
  double avcon = 0., vismud = 0., visfac = 0.;
  std::vector<double> zbr, zbratu, zbratv, sgzuu, sgzvv, stbxo, stbyo, stbx, stby;
  // explicit momentum producer (CALEXP2T): the static part, layer k (0-based)
  // of a layer array at [k*(lc+2) + L], and the SAVEd / module layer arrays
  // kept between calls (zero before the first), with the wet set of the
  // previous call (its newly dry cells are LDRY)
  bool mom = false;
  int mkc = 0, mld = 0;
  std::vector<double> fcorc, dydi, dxdj, scax, scay, saax, saay, stcuv, sdx, sdy;
  std::vector<double> msgzu, msgzv, mfsgzu, mfsgzv;
  std::vector<int> lhdmf, lnwc, lsec, lbcs, lberc, lbnrc;
  std::vector<double> fuhu, fvhu, fvhv, fuhv, cac, fcax, fcay, fx, fy;
  std::vector<int> mwet_prev;
};

namespace {

template <class Fn>
void for_domains(const oracle_ctx *c, Fn &&fn) {
  // !$OMP PARALLEL DO over ND=1,NOPTIMAL with LF=2+(ND-1)*LDMOPT (calpuv2c.f90:164-167)
  const int nopt = c->noptimal, ldm = c->ldmopt, la = c->la;
#pragma omp parallel for num_threads(nopt) schedule(static, 1) if (nopt > 1)
  for (int nd = 1; nd <= nopt; ++nd) {
    const int lf = 2 + (nd - 1) * ldm;
    const int ll = std::min(lf + ldm - 1, la);
    for (int L = lf; L <= ll; ++L) fn(L);
  }
}

template <class T>
void copy1(std::vector<T> &dst, const T *src, int lc) {
  dst.assign(lc + 2, T(0));
  if (src)
    for (int L = 1; L <= lc; ++L) dst[L] = src[L - 1];
}

// CONGRAD body (congrad.f90:54-187) on the context's scaled system.  With
// channels (chan = true) it is CONGRADC (congradc.f90:1-207): the same
// iteration plus the host-guest couplings CCCCHH, added as written to the
// initial residual (:59-77) and to A*p (:99-116); with `consistent` A*p takes
// -CCCCHH instead (the operator of the residual).  p is the caller's 1-based
// P. Returns 0 or EFDC_XM_CG_MAXITER / NONFINITE.
int congrad(oracle_ctx *c, F<double> P, double rsqm, int iterm, int *iters_out,
            double *rsq_out, bool chan = false, bool consistent = false) {
  const int la = c->la;
  const int *LNC = c->lnc.data(), *LSC = c->lsc.data(), *LEC = c->lec.data(),
            *LWC = c->lwc.data();
  double *PCG = c->pcg.data(), *PN = c->pnv.data(), *PE = c->pev.data(),
         *PW = c->pwv.data(), *PS = c->psv.data(), *RCG = c->rcg.data(),
         *APCG = c->apcg.data(), *TMPCG = c->tmpcg.data();
  const double *CCC = c->ccc.data(), *CCS = c->ccs.data(), *CCN = c->ccn.data(),
               *CCW = c->ccw.data(), *CCE = c->cce.data(),
               *CCCI = c->ccci.data(), *FPTMP = c->fptmp.data();

  // :54-77  neighbour gathers of P, then the initial residual
  for_domains(c, [&](int L) {
    PN[L] = P[LNC[L]];
    PE[L] = P[LEC[L]];
    PW[L] = P[LWC[L]];
    PS[L] = P[LSC[L]];
  });
  for_domains(c, [&](int L) {
    RCG[L] = FPTMP[L] - CCC[L] * P[L] - CCN[L] * PN[L] - CCS[L] * PS[L] -
             CCW[L] * PW[L] - CCE[L] * PE[L];
  });
  const Channels &ch = c->ch;
  if (chan)  // congradc.f90:59-77
    for (int k = 0; k < ch.n; ++k) {
      const int LH = ch.lh[k];
      if (ch.typ[k] == 1) {
        const int LU = ch.lu[k];
        RCG[LU] = RCG[LU] + ch.chh[k] * P[LH];
        RCG[LH] = RCG[LH] + ch.chh[k] * P[LU];
      }
      if (ch.typ[k] == 2) {
        const int LV = ch.lv[k];
        RCG[LV] = RCG[LV] + ch.chh[k] * P[LH];
        RCG[LH] = RCG[LH] + ch.chh[k] * P[LV];
      }
    }
  // :79-88
  for (int L = 2; L <= la; ++L) PCG[L] = RCG[L] * CCCI[L];
  double RPCG = 0.;
  for (int L = 2; L <= la; ++L) RPCG = RPCG + RCG[L] * PCG[L];
  *rsq_out = 0.;
  if (RPCG == 0.0) {  // :88 "DS-INTL SINGLE LINE": ITER is left untouched
    *iters_out = 0;
    return EFDC_XM_OK;
  }

  double RSQ = 0.;
  int iter;
  const int nopt = c->noptimal, ldm = c->ldmopt;
  for (iter = 1; iter <= iterm; ++iter) {  // :91
    double PAPCG = 0., ALPHA = 0., RPCGN = 0., BETA = 0.;
#pragma omp parallel num_threads(nopt) if (nopt > 1)
    {
#pragma omp for schedule(static, 1)
      for (int nd = 1; nd <= nopt; ++nd) {  // :93-105
        const int lf = 2 + (nd - 1) * ldm, ll = std::min(lf + ldm - 1, la);
        for (int L = lf; L <= ll; ++L) {
          PN[L] = PCG[LNC[L]];
          PE[L] = PCG[LEC[L]];
          PW[L] = PCG[LWC[L]];
          PS[L] = PCG[LSC[L]];
        }
      }
#pragma omp for schedule(static, 1)
      for (int nd = 1; nd <= nopt; ++nd) {  // :107-116
        const int lf = 2 + (nd - 1) * ldm, ll = std::min(lf + ldm - 1, la);
        for (int L = lf; L <= ll; ++L)
          APCG[L] = CCC[L] * PCG[L] + CCS[L] * PS[L] + CCN[L] * PN[L] +
                    CCW[L] * PW[L] + CCE[L] * PE[L];
      }
#pragma omp single
      {  // :118-125 serial dot "to prevent roundoff error"
        if (chan)  // congradc.f90:99-116
          for (int k = 0; k < ch.n; ++k) {
            const int LH = ch.lh[k];
            const double h = consistent ? -ch.chh[k] : ch.chh[k];
            if (ch.typ[k] == 1) {
              const int LU = ch.lu[k];
              APCG[LU] = APCG[LU] + h * PCG[LH];
              APCG[LH] = APCG[LH] + h * PCG[LU];
            }
            if (ch.typ[k] == 2) {
              const int LV = ch.lv[k];
              APCG[LV] = APCG[LV] + h * PCG[LH];
              APCG[LH] = APCG[LH] + h * PCG[LV];
            }
          }
        PAPCG = 0.;
        for (int L = 2; L <= la; ++L) PAPCG = PAPCG + APCG[L] * PCG[L];
        ALPHA = RPCG / PAPCG;
      }
#pragma omp for schedule(static, 1)
      for (int nd = 1; nd <= nopt; ++nd) {  // :127-137
        const int lf = 2 + (nd - 1) * ldm, ll = std::min(lf + ldm - 1, la);
        for (int L = lf; L <= ll; ++L) {
          P[L] = P[L] + ALPHA * PCG[L];
          RCG[L] = RCG[L] - ALPHA * APCG[L];
          TMPCG[L] = CCCI[L] * RCG[L];
        }
      }
#pragma omp single
      {  // :139-149
        RPCGN = 0.;
        RSQ = 0.;
        for (int L = 2; L <= la; ++L) {
          RPCGN = RPCGN + RCG[L] * TMPCG[L];
          RSQ = RSQ + RCG[L] * RCG[L];
        }
        BETA = RPCGN / RPCG;
        RPCG = RPCGN;
      }
      if (RSQ > rsqm) {  // :151-162
#pragma omp for schedule(static, 1)
        for (int nd = 1; nd <= nopt; ++nd) {
          const int lf = 2 + (nd - 1) * ldm, ll = std::min(lf + ldm - 1, la);
          for (int L = lf; L <= ll; ++L) PCG[L] = TMPCG[L] + BETA * PCG[L];
        }
      }
    }
    if (!std::isfinite(RSQ) || !std::isfinite(ALPHA)) {
      *iters_out = iter;
      *rsq_out = RSQ;
      return EFDC_XM_NONFINITE;
    }
    if (RSQ <= rsqm) break;  // :165-167
  }
  *rsq_out = RSQ;
  if (RSQ > rsqm) {  // :171-184 (the reference dumps and STOPs)
    *iters_out = iterm;
    return EFDC_XM_CG_MAXITER;
  }
  *iters_out = iter;  // IDRYTBP = ITER (:187)
  return EFDC_XM_OK;
}

// SUBCHAN (subchan.f90:1-124): per channel NMD in order, the activity test,
// the implicit coefficients CCCCHU, CCCCHV, CCCCHH, and their entries in CC
// and FP of the host and guest cells.  RLAMN = QCHERR, DE_T = DELT.
void subchan(oracle_ctx *c, double G, double DE_T, double HDRY, double RLAMN,
             F<const double> H1P, F<const double> HP, double *CC, double *FP) {
  Channels &ch = c->ch;
  const double RLAMO = 1. - RLAMN;
  const double *BELV = c->belv.data(), *P1 = c->p1.data();
  for (int k = 0; k < ch.n; ++k) {
    ch.cu[k] = 0.0;
    ch.cv[k] = 0.0;
    ch.chh[k] = 0.0;
    const int LHOST = ch.lh[k], LCHNU = ch.lu[k], LCHNV = ch.lv[k];
    if (ch.typ[k] == 1) {  // :29-62 x-direction channel
      ch.iact[k] = 0;
      const double SRFHOST = H1P[LHOST] + BELV[LHOST];
      const double SRFCHAN = H1P[LCHNU] + BELV[LCHNU];
      if (SRFCHAN > SRFHOST)
        if (H1P[LCHNU] > HDRY) ch.iact[k] = 1;
      if (SRFHOST > SRFCHAN)
        if (H1P[LHOST] > HDRY) ch.iact[k] = 1;
      if (HP[LHOST] <= 0.0 || HP[LCHNU] <= 0.0)
        if (ch.iact[k] == 1) ch.iact[k] = 0;
      if (ch.iact[k] == 1) {
        const double WCHAN = ch.dxp[LCHNU];
        const double RLCHN = 0.5 * ch.dyp[LCHNU] + ch.len[k];
        double HCHAN = 0.5 * ch.dyp[LCHNU] * H1P[LCHNU] + ch.len[k] * H1P[LHOST];
        HCHAN = HCHAN / RLCHN;
        if (HCHAN > 0.) {
          const double TMPVAL = ch.fric[k] * DE_T / (HCHAN * HCHAN * WCHAN);
          ch.cu[k] = 1. / (1. + TMPVAL * std::fabs(ch.qut[k]));
          ch.cv[k] = DE_T * HCHAN * WCHAN / RLCHN;
        }
      }
    }
    if (ch.typ[k] == 2) {  // :64-101 y-direction channel
      int IHCHMX = 0, IHCHMN = 0;
      double HCHNMX = 0., HCHNMN = 0.;
      ch.iact[k] = 0;
      const double SRFHOST = H1P[LHOST] + BELV[LHOST];
      const double SRFCHAN = H1P[LCHNV] + BELV[LCHNV];
      if (SRFCHAN > SRFHOST)
        if (H1P[LCHNV] > HDRY) {
          HCHNMX = -H1P[LCHNV];
          IHCHMX = 1;
          ch.iact[k] = 1;
        }
      if (SRFHOST > SRFCHAN)
        if (H1P[LHOST] > HDRY) {
          HCHNMN = H1P[LHOST];
          IHCHMN = 1;
          ch.iact[k] = 1;
        }
      // :84 tests HP(LCHNU) for the y-direction channel too, as written
      if (HP[LHOST] <= 0.0 || HP[LCHNU] <= 0.0)
        if (ch.iact[k] == 1) ch.iact[k] = 0;
      if (ch.iact[k] == 1) {
        const double WCHAN = ch.dyp[LCHNV];
        const double RLCHN = 0.5 * ch.dxp[LCHNV] + ch.len[k];
        double HCHAN = 0.5 * ch.dxp[LCHNV] * H1P[LCHNV] + ch.len[k] * H1P[LHOST];
        HCHAN = HCHAN / RLCHN;
        if (IHCHMX == 1) HCHAN = std::max(HCHAN, HCHNMX);
        if (IHCHMN == 1) HCHAN = std::min(HCHAN, HCHNMN);
        if (HCHAN > 0.) {
          const double TMPVAL = ch.fric[k] * DE_T / (HCHAN * HCHAN * WCHAN);
          ch.cu[k] = 1. / (1. + TMPVAL * std::fabs(ch.qvt[k]));
          ch.cv[k] = DE_T * HCHAN * WCHAN / RLCHN;
        }
      }
    }
    // :104-119
    CC[LHOST] = CC[LHOST] + G * RLAMN * RLAMN * ch.cu[k] * ch.cv[k];
    ch.chh[k] = G * RLAMN * RLAMN * ch.cu[k] * ch.cv[k];
    if (ch.typ[k] == 1) {
      CC[LCHNU] = CC[LCHNU] + G * RLAMN * RLAMN * ch.cu[k] * ch.cv[k];
      const double TMPVAL = G * (RLAMO + RLAMN * ch.cu[k]) * ch.qut[k] -
                            G * RLAMN * RLAMO * ch.cu[k] * ch.cv[k] * (P1[LHOST] - P1[LCHNU]);
      FP[LHOST] = FP[LHOST] + TMPVAL;
      FP[LCHNU] = FP[LCHNU] - TMPVAL;
    }
    if (ch.typ[k] == 2) {
      CC[LCHNV] = CC[LCHNV] + G * RLAMN * RLAMN * ch.cu[k] * ch.cv[k];
      const double TMPVAL = G * (RLAMO + RLAMN * ch.cu[k]) * ch.qvt[k] -
                            G * RLAMN * RLAMO * ch.cu[k] * ch.cv[k] * (P1[LHOST] - P1[LCHNV]);
      FP[LHOST] = FP[LHOST] + TMPVAL;
      FP[LCHNV] = FP[LCHNV] - TMPVAL;
    }
  }
}

}  // namespace

extern "C" {

oracle_ctx *oracle_create(const efdc_xm_grid *g, int nthreads, int noptimal_cap) {
  if (!g || g->la < 2 || g->lc != g->la + 1) return nullptr;
  oracle_ctx *c = new oracle_ctx();
  c->la = g->la;
  c->lc = g->lc;
  c->nthreads = std::max(1, nthreads);
  // calpuv2c.f90:61-62
  c->noptimal = std::min(std::min(c->nthreads, std::max(1, noptimal_cap)),
                         std::max(c->la / 100, 1));
  c->ldmopt = int(double(c->la - 1) / double(c->noptimal)) + 1;
  const int lc = c->lc;
  copy1(c->lnc, g->lnc, lc);
  copy1(c->lsc, g->lsc, lc);
  copy1(c->lec, g->lec, lc);
  copy1(c->lwc, g->lwc, lc);
  copy1(c->dxyp, g->dxyp, lc);
  copy1(c->dxyip, g->dxyip, lc);
  copy1(c->dxiu, g->dxiu, lc);
  copy1(c->dyiu, g->dyiu, lc);
  copy1(c->dxiv, g->dxiv, lc);
  copy1(c->dyiv, g->dyiv, lc);
  copy1(c->dxyu, g->dxyu, lc);
  copy1(c->dxyv, g->dxyv, lc);
  copy1(c->hruo, g->hruo, lc);
  copy1(c->hrvo, g->hrvo, lc);
  copy1(c->subo, g->subo, lc);
  copy1(c->svbo, g->svbo, lc);
  copy1(c->sbxo, g->sbxo, lc);
  copy1(c->sbyo, g->sbyo, lc);
  copy1(c->belv, g->belv, lc);
  c->mtide = g->mtide;
  c->tcp.assign(g->tcp ? g->tcp : nullptr, g->tcp ? g->tcp + g->mtide : nullptr);
  for (int s = 0; s < 4; ++s) {
    const efdc_xm_obc &o = g->obc[s];
    Side &d = c->side[s];
    d.n = o.n;
    d.l.assign(o.l, o.l + o.n);
    d.ispb.assign(o.ispb, o.ispb + o.n);
    d.pcb.assign(size_t(o.n) * std::max(g->mtide, 0), 0.0);
    d.psb.assign(size_t(o.n) * std::max(g->mtide, 0), 0.0);
    for (int m = 0; m < g->mtide; ++m)
      for (int ll = 0; ll < o.n; ++ll) {
        d.pcb[size_t(m) * o.n + ll] = o.pcb ? o.pcb[size_t(m) * o.ld + ll] : 0.0;
        d.psb[size_t(m) * o.n + ll] = o.psb ? o.psb[size_t(m) * o.ld + ll] : 0.0;
      }
  }
  // LOBCS order: S, W, E, N
  const int order[4] = {EFDC_XM_OBC_S, EFDC_XM_OBC_W, EFDC_XM_OBC_E, EFDC_XM_OBC_N};
  for (int k = 0; k < 4; ++k)
    for (int l : c->side[order[k]].l) c->lobcs.push_back(l);

  const size_t n = size_t(lc) + 2;
  for (auto *v : {&c->fp1, &c->fp, &c->fuhdye, &c->fvhdxe, &c->cs, &c->cw,
                  &c->ce, &c->cn, &c->cc, &c->ccs, &c->ccw, &c->cce, &c->ccn,
                  &c->ccc, &c->ccci, &c->fptmp, &c->rcx, &c->rcy, &c->sub1,
                  &c->svb1, &c->fsgzu, &c->fsgzv, &c->uhdy1e, &c->vhdx1e,
                  &c->pcg, &c->pnv, &c->pev, &c->pwv, &c->psv, &c->rcg,
                  &c->apcg, &c->tmpcg})
    v->assign(n, 0.0);
  c->oldmask.assign(n, 0);
  // first-call initialisation (calpuv2c.f90:97-123)
  std::fill(c->rcx.begin(), c->rcx.end(), 1.0);
  std::fill(c->rcy.begin(), c->rcy.end(), 1.0);
  c->rcx[1] = c->rcy[1] = 0.;
  c->rcx[lc] = c->rcy[lc] = 0.;
  std::fill(c->cc.begin(), c->cc.end(), 1.0);
  std::fill(c->fsgzu.begin(), c->fsgzu.end(), 1.0);
  std::fill(c->fsgzv.begin(), c->fsgzv.end(), 1.0);
  for (int L = 2; L <= c->la; ++L) {
    c->fsgzu[L] = 0.5 / c->dxyu[L];
    c->fsgzv[L] = 0.5 / c->dxyv[L];
  }
  return c;
}

void oracle_destroy(oracle_ctx *c) { delete c; }

int oracle_noptimal(const oracle_ctx *c) { return c ? c->noptimal : 0; }

int oracle_step(oracle_ctx *c, const efdc_xm_params *prm, efdc_xm_fields *f,
                efdc_xm_stats *st) {
  efdc_xm_stats dummy;
  if (!st) st = &dummy;
  std::memset(st, 0, sizeof(*st));
  const int la = c->la, lc = c->lc;
  const int *LNC = c->lnc.data(), *LSC = c->lsc.data(), *LEC = c->lec.data(),
            *LWC = c->lwc.data();
  const double *DXYP = c->dxyp.data(), *DXYIP = c->dxyip.data(),
               *DXIU = c->dxiu.data(), *DYIU = c->dyiu.data(),
               *DXIV = c->dxiv.data(), *DYIV = c->dyiv.data(),
               *DXYU = c->dxyu.data(), *DXYV = c->dxyv.data(),
               *HRUO = c->hruo.data(), *HRVO = c->hrvo.data(),
               *SUBO = c->subo.data(), *SVBO = c->svbo.data(),
               *SBXO = c->sbxo.data(), *SBYO = c->sbyo.data(),
               *BELV = c->belv.data();
  double *FP1 = c->fp1.data(), *FP = c->fp.data(), *FUHDYE = c->fuhdye.data(),
         *FVHDXE = c->fvhdxe.data(), *CS = c->cs.data(), *CW = c->cw.data(),
         *CE = c->ce.data(), *CN = c->cn.data(), *CC = c->cc.data(),
         *CCS = c->ccs.data(), *CCW = c->ccw.data(), *CCE = c->cce.data(),
         *CCN = c->ccn.data(), *CCC = c->ccc.data(), *CCCI = c->ccci.data(),
         *FPTMP = c->fptmp.data(), *RCX = c->rcx.data(), *RCY = c->rcy.data(),
         *SUB1 = c->sub1.data(), *SVB1 = c->svb1.data(),
         *FSGZU = c->fsgzu.data(), *FSGZV = c->fsgzv.data(),
         *UHDY1E = c->uhdy1e.data(), *VHDX1E = c->vhdx1e.data();
  int *OLDMASK = c->oldmask.data();

  F<double> P{f->p}, HP{f->hp}, H1P{f->h1p}, HU{f->hu}, HV{f->hv},
      UHDYE{f->uhdye}, VHDXE{f->vhdxe}, SUB{f->sub}, SVB{f->svb}, SBX{f->sbx},
      SBY{f->sby};
  F<int32_t> LMASKDRY{f->lmaskdry}, ISCDRY{f->iscdry},
      LOPENBCDRY{f->lopenbcdry}, NATDRY{f->natdry};
  std::vector<double> zeros(size_t(lc) + 1, 0.0);
  auto cin = [&](const double *p) { return F<const double>{p ? p : zeros.data()}; };
  F<const double> FCAXE = cin(f->fcaxe), FCAYE = cin(f->fcaye), FXE = cin(f->fxe),
                  FYE = cin(f->fye), TSX = cin(f->tsx), TSY = cin(f->tsy),
                  TBX = cin(f->tbx), TBY = cin(f->tby), QSUME = cin(f->qsume);
  // implicit drag inputs (ISITB >= 1, ISVEG > 0): U(L,KSZU(L)), V(L,KSZV(L)),
  // VU, UV, STBX, STBY, FXVEGE, FYVEGE
  F<const double> UBOT = cin(f->ubot), VBOT = cin(f->vbot), VU = cin(f->vu), UV = cin(f->uv),
                  STBX = cin(f->stbx), STBY = cin(f->stby), FXVEGE = cin(f->fxvege),
                  FYVEGE = cin(f->fyvege);
  std::vector<double> qdw_local, vdw_local, uhe_l, vhe_l, hpi_l, hui_l, hvi_l;
  auto opt = [&](double *p, std::vector<double> &store) {
    if (p) return F<double>{p};
    store.assign(size_t(lc) + 1, 0.0);
    return F<double>{store.data()};
  };
  F<double> QDWASTE = opt(f->qdwaste, qdw_local), VDWASTE = opt(f->vdwaste, vdw_local),
            UHE = opt(f->uhe, uhe_l), VHE = opt(f->vhe, vhe_l),
            HPI = opt(f->hpi, hpi_l), HUI = opt(f->hui, hui_l),
            HVI = opt(f->hvi, hvi_l);

  const double G = prm->g;
  const double GI = 1. / G;  // aaefdc.f90:648
  // CALPUV2C (ISTL = 0 here), or CALPUV9C(ISTL_) of the three-time-level scheme
  const int ISTL = prm->tl3_istl;
  const bool tl3 = ISTL != 0;
  if (tl3 && ((ISTL != 2 && ISTL != 3) || !f->p1 || !f->h2p || !f->uhdy1e || !f->vhdx1e ||
              !f->uhdy2e || !f->vhdx2e || !f->h1u || !f->h1v)) {
    st->status = EFDC_XM_BAD_ARGUMENT;
    return EFDC_XM_BAD_ARGUMENT;
  }
  // calpuv2c.f90:128-136; calpuv9c.f90:105-111 (DELT = DT2 or DT as passed:
  // DELTD2 = DT = DT2/2, or DT/2)
  const double DELT = prm->delt;
  const double DELTD2 = 0.5 * DELT;
  const double DELTI = 1. / DELT;
  const double HDRY = prm->hdry;
  const int ISDRY = prm->isdry, NDRYSTP = prm->ndrystp;
  const double RITB1 = prm->ritb1, SNLT = prm->snlt;
  const int ISITB = prm->isitb, ISVEG = prm->isveg;
  const double RITB = prm->ritb;
  // calpuv2c.f90:222-243 (calpuv9c.f90:220-240): the implicit bottom drag with
  // vegetation, or the vegetation drag alone, of cell L; HUI(L) = 1./HU(L) as
  // the previous step left it (:902-906)
  auto implicit_drag = [&](int L) {
    if (ISITB >= 1) {
      double TMPX = 1.0, TMPY = 1.0;
      if (UHE[L] != 0.0) TMPX = UBOT[L] * HU[L] / UHE[L];
      if (VHE[L] != 0.0) TMPY = VBOT[L] * HV[L] / VHE[L];
      const double HUIL = 1. / HU[L], HVIL = 1. / HV[L];
      RCX[L] = 1. / (1. + TMPX * RITB * DELT * HUIL * STBX[L] *
                              std::sqrt(VU[L] * VU[L] + UBOT[L] * UBOT[L]) +
                     DELT * FXVEGE[L]);
      RCY[L] = 1. / (1. + TMPY * RITB * DELT * HVIL * STBY[L] *
                              std::sqrt(UV[L] * UV[L] + VBOT[L] * VBOT[L]) +
                     DELT * FYVEGE[L]);
      FUHDYE[L] = FUHDYE[L] * RCX[L];
      FVHDXE[L] = FVHDXE[L] * RCY[L];
    } else if (ISVEG > 0) {
      RCX[L] = 1. / (1. + DELT * FXVEGE[L]);
      RCY[L] = 1. / (1. + DELT * FYVEGE[L]);
      FUHDYE[L] = FUHDYE[L] * RCX[L];
      FVHDXE[L] = FVHDXE[L] * RCY[L];
    }
  };
  const bool baro = prm->bsc > 1.E-6;
  if (baro && (c->kc < 1 || !f->b || (tl3 && (!f->fpgxe || !f->fpgye)))) {
    st->status = EFDC_XM_BAD_ARGUMENT;
    return EFDC_XM_BAD_ARGUMENT;
  }
  if (baro) {  // :161 CALL CALEBI (calebi.f90:73-120, standard sigma, KSZ = 1)
    const size_t ldb = size_t(f->b_ld), ldl = size_t(lc) + 2;
    for (int L = 2; L <= la; ++L) {
      if (ISDRY > 0 && !f->lmaskdry[L - 1]) continue;  // LWET of the last step
      double DBK = 0., BEC = 0., BI1C = 0., BI2C = 0.;
      for (int K = c->kc; K >= 1; --K) {
        const double DZCC = c->dzc[size_t(K - 1) * ldl + L];
        const double DZCB = DZCC * f->b[size_t(K - 1) * ldb + (L - 1)];
        DBK = DBK + DZCB;  // :94-98
        const double BK = DBK - 0.5 * DZCB;
        BEC = BEC + DZCB;  // :100-108
        const double DZCBK = DZCC * BK;
        BI1C = BI1C + DZCBK;
        BI2C = BI2C + DZCBK + c->zz[size_t(K - 1) * ldl + L] * DZCB;
      }
      c->bi1[L] = BI1C;  // BI1W = BI1S (:110-118)
      c->bi2[L] = BI2C;
      c->be[L] = BEC;
    }
  }
  const double GP = prm->gp;
  const double *BI1 = c->bi1.data(), *BI2 = c->bi2.data(), *BE = c->be.data();
  const int max_sweeps = prm->max_sweeps > 0 ? prm->max_sweeps : 500;

  int NCORDRY = 0;
  Channels &ch = c->ch;
  const bool chans = ch.n > 0;
  const double RLAMN = prm->qcherr, RLAMO = 1. - RLAMN;  // :353-354
  if (chans) {
    if (!f->qchanu || !f->qchanv || !f->qchanun || !f->qchanvn) {
      st->status = EFDC_XM_BAD_ARGUMENT;
      return EFDC_XM_BAD_ARGUMENT;
    }
    for (int k = 0; k < ch.n; ++k) {
      if (!tl3) {  // :139-145
        ch.qut[k] = f->qchanu[k];
        ch.qvt[k] = f->qchanv[k];
      } else {  // calpuv9c.f90:128-141
        ch.qut[k] = f->qchanun[k];
        ch.qvt[k] = f->qchanvn[k];
        if (ISTL == 3) {
          f->qchanun[k] = f->qchanu[k];
          f->qchanvn[k] = f->qchanv[k];
        }
      }
    }
    // P1 as SUBCHAN and the exchange read it: P at entry (:259, and
    // calpuv9c.f90:302 for ISTL_ = 3), the caller's P1 for ISTL_ = 2
    for (int L = 1; L <= lc; ++L) c->p1[L] = (ISTL == 2) ? f->p1[L - 1] : P[L];
  }
  // :150-157
  if (ISDRY > 0)
    for (int L : c->lobcs) LOPENBCDRY[L] = 0;

  std::vector<int> nnatdry_flag(size_t(lc) + 1, 0);

  // Three time levels: the caller's arrays, and HUTMP/HVTMP, the face depths
  // of the coefficients (HU, HV in CALPUV2C; HUTMP(1), HUTMP(LC) stay 0,
  // varzeroreal.f90:249)
  std::vector<double> hutmp(size_t(lc), 0.0), hvtmp(size_t(lc), 0.0);
  F<double> HUT{hutmp.data()}, HVT{hvtmp.data()};
  F<double> P1T{f->p1}, H2P{f->h2p}, U1{f->uhdy1e}, V1{f->vhdx1e}, U2{f->uhdy2e},
      V2{f->vhdx2e}, H1U{f->h1u}, H1V{f->h1v}, FPGX{f->fpgxe}, FPGY{f->fpgye};
  F<const double> TSX1 = cin(f->tsx1), TSY1 = cin(f->tsy1), TBX1 = cin(f->tbx1),
                  TBY1 = cin(f->tby1);
  const F<const double> HUc{tl3 ? HUT.b : HU.b}, HVc{tl3 ? HVT.b : HV.b};

  if (tl3) {  // ---- CALPUV9C up to 1000 CONTINUE (calpuv9c.f90:128-311) ----
    if (ISDRY > 0 && NDRYSTP < 0)  // :154-160
      for (int L = 2; L <= la; ++L) QDWASTE[L] = 0.;
    for_domains(c, [&](int L) {  // :164-204
      if (baro) {  // external density gradients, blended with the last ones
        const int LW = LWC[L], LS = LSC[L];
        FPGX[L] = prm->rold * FPGX[L] +
                  prm->rnew * (-SBX[L] * HU[L] * GP *
                               ((BI2[L] + BI2[LW]) * (HP[L] - HP[LW]) +
                                2.0 * HU[L] * (BI1[L] - BI1[LW]) +
                                (BE[L] + BE[LW]) * (BELV[L] - BELV[LW])));
        FPGY[L] = prm->rold * FPGY[L] +
                  prm->rnew * (-SBY[L] * HV[L] * GP *
                               ((BI2[L] + BI2[LS]) * (HP[L] - HP[LS]) +
                                2.0 * HV[L] * (BI1[L] - BI1[LS]) +
                                (BE[L] + BE[LS]) * (BELV[L] - BELV[LS])));
      }
      if (ISTL == 2) {
        HUT[L] = 0.5 * (HU[L] + H1U[L]);
        HVT[L] = 0.5 * (HV[L] + H1V[L]);
      } else {
        HUT[L] = HU[L];
        HVT[L] = HV[L];
      }
    });
    for_domains(c, [&](int L) {  // :206-222 explicit transports from level n-1
      const int LS = LSC[L], LW = LWC[L];
      const double FPGXE = baro ? FPGX[L] : 0., FPGYE = baro ? FPGY[L] : 0.;
      FUHDYE[L] = U1[L] - DELTD2 * SUB[L] * HRUO[L] * HUT[L] * (P1T[L] - P1T[LW]) +
                  SUB[L] * DELT * DXIU[L] *
                      (DXYU[L] * (TSX1[L] - RITB1 * TBX1[L]) + FCAXE[L] + FPGXE -
                       SNLT * FXE[L]);
      FVHDXE[L] = V1[L] - DELTD2 * SVB[L] * HRVO[L] * HVT[L] * (P1T[L] - P1T[LS]) +
                  SVB[L] * DELT * DYIV[L] *
                      (DXYV[L] * (TSY1[L] - RITB1 * TBY1[L]) - FCAYE[L] + FPGYE -
                       SNLT * FYE[L]);
      implicit_drag(L);  // :220-240
    });
    if (ISDRY > 0)  // :246-262
      for_domains(c, [&](int L) {
        ISCDRY[L] = 0;
        SUB1[L] = SUB[L];
        SVB1[L] = SVB[L];
        SUB[L] = SUBO[L];
        SVB[L] = SVBO[L];
        SBX[L] = SBXO[L];
        SBY[L] = SBYO[L];
        OLDMASK[L] = LMASKDRY[L];
      });
    for_domains(c, [&](int L) {  // :268-280
      const double C1 = 0.5 * G;
      const int LE = LEC[L], LN = LNC[L];
      FP1[L] = DELTI * DXYP[L] * P1T[L] - C1 * (U1[LE] - U1[L] + V1[LN] - V1[L]);
    });
    if (ISTL == 3)  // :282-311 advance the time levels (the 2D ones)
      for_domains(c, [&](int L) {
        if (prm->nctbc == 1) {
          UHDYE[L] = 0.5 * UHDYE[L];
          VHDXE[L] = 0.5 * VHDXE[L];
        }
        U2[L] = U1[L];
        V2[L] = V1[L];
        U1[L] = UHDYE[L];
        V1[L] = VHDXE[L];
        P1T[L] = P[L];
        H1U[L] = HU[L];
        H1V[L] = HV[L];
        H2P[L] = H1P[L];
        H1P[L] = HP[L];
      });
  } else  // ---- first domain loop (:164-293) ----
  for_domains(c, [&](int L) {
    if (ISDRY > 0) {  // :172-190
      ISCDRY[L] = 0;
      SUB1[L] = SUB[L];
      SVB1[L] = SVB[L];
      OLDMASK[L] = LMASKDRY[L];
      if (NDRYSTP < 0 && prm->isbal > 0) QDWASTE[L] = 0.;
    }
    {  // :214-220 explicit external transports
      const int LS = LSC[L], LW = LWC[L];
      double FPGXE = 0., FPGYE = 0.;
      if (baro) {  // :192-201 external density gradients (IGRIDV = 0)
        FPGXE = -SBX[L] * HU[L] * GP *
                ((BI2[L] + BI2[LW]) * (HP[L] - HP[LW]) + 2.0 * HU[L] * (BI1[L] - BI1[LW]) +
                 (BE[L] + BE[LW]) * (BELV[L] - BELV[LW]));
        FPGYE = -SBY[L] * HV[L] * GP *
                ((BI2[L] + BI2[LS]) * (HP[L] - HP[LS]) + 2.0 * HV[L] * (BI1[L] - BI1[LS]) +
                 (BE[L] + BE[LS]) * (BELV[L] - BELV[LS]));
      }
      FUHDYE[L] = UHDYE[L] - DELTD2 * SUB[L] * HRUO[L] * HU[L] * (P[L] - P[LW]) +
                  SUB[L] * DELT * DXIU[L] *
                      (DXYU[L] * (TSX[L] - RITB1 * TBX[L]) + FCAXE[L] + FPGXE -
                       SNLT * FXE[L]);
      FVHDXE[L] = VHDXE[L] - DELTD2 * SVB[L] * HRVO[L] * HV[L] * (P[L] - P[LS]) +
                  SVB[L] * DELT * DYIV[L] *
                      (DXYV[L] * (TSY[L] - RITB1 * TBY[L]) - FCAYE[L] + FPGYE -
                       SNLT * FYE[L]);
    }
    implicit_drag(L);  // :222-243
    if (ISDRY > 0) {  // :246-253
      SUB[L] = SUBO[L];
      SVB[L] = SVBO[L];
      SBX[L] = SBXO[L];
      SBY[L] = SBYO[L];
    }
    // :256-266 advance the external variables (the 2D ones this library owns)
    UHDY1E[L] = UHDYE[L];
    VHDX1E[L] = VHDXE[L];
    H1P[L] = HP[L];
    {  // :282-290
      const double C1 = 0.5 * G;
      const int LE = LEC[L], LN = LNC[L];
      FP1[L] = DELTI * DXYP[L] * P[L] -
               C1 * (UHDYE[LE] - UHDYE[L] + VHDXE[LN] - VHDXE[L]);
    }
  });

  int iters_total = 0, solves = 0, last_iters = 0, status = EFDC_XM_OK;
  double last_rsq = 0., last_ccmnm = 0.;

  for (;;) {  // ---- 1000 CONTINUE (:298) ----
    // :306-344 new-time-level continuity terms and the coefficients
    for_domains(c, [&](int L) {
      double C1 = 0.5 * G;
      const int LE = LEC[L], LN = LNC[L];
      FP[L] = FP1[L] - C1 * (SUB[LE] * FUHDYE[LE] - SUB[L] * FUHDYE[L] +
                             SVB[LN] * FVHDXE[LN] - SVB[L] * FVHDXE[L] -
                             2.0 * QSUME[L]);
      C1 = -0.5 * DELTD2 * G;
      CS[L] = C1 * SVB[L] * HRVO[L] * RCY[L] * HVc[L];  // HVTMP in CALPUV9C (calpuv9c.f90:369-379)
      CW[L] = C1 * SUB[L] * HRUO[L] * RCX[L] * HUc[L];
      CE[L] = C1 * SUB[LE] * HRUO[LE] * RCX[LE] * HUc[LE];
      CN[L] = C1 * SVB[LN] * HRVO[LN] * RCY[LN] * HVc[LN];
      CC[L] = DELTI * DXYP[L] - CS[L] - CW[L] - CE[L] - CN[L];
    });

    // :349 SETOPENBC(DELTD2,DELTI,HU,HV)  (setopenbc.f90:1-206); CALPUV9C passes
    // HUTMP, HVTMP (calpuv9c.f90:389)
    if (!c->lobcs.empty()) {
      const double D_LTD2 = DELTD2, DE_TI = DELTI;
      const double HDRY2 = 0.2 * HDRY;
      const double TN = prm->tn;
      std::vector<double> CCCOS(size_t(std::max(c->mtide, 1))),
          SSSIN(size_t(std::max(c->mtide, 1)));
      for (int m = 0; m < c->mtide; ++m) {  // :24-29
        double TM = std::fmod(TN, c->tcp[m]);
        TM = prm->pi2 * TM / c->tcp[m];
        CCCOS[m] = std::cos(TM);
        SSSIN[m] = std::sin(TM);
      }
      auto target = [&](const Side &s, const double *pser, int ll, int L) {
        // FP(L)=PSERT+...(series part supplied by the caller), then :47-52
        double v = pser ? pser[ll] : 0.0;
        for (int m = 0; m < c->mtide; ++m) {
          const double TC = CCCOS[m], TS = SSSIN[m];
          v = v + s.pcb[size_t(m) * s.n + ll] * TC + s.psb[size_t(m) * s.n + ll] * TS;
        }
        (void)L;
        return v;
      };
      {  // WEST :32-74
        const Side &s = c->side[EFDC_XM_OBC_W];
        for (int ll = 0; ll < s.n; ++ll) {
          const int L = s.l[ll];
          CC[L] = DELTI * DXYP[L];
          CS[L] = 0.; CW[L] = 0.; CE[L] = 0.; CN[L] = 0.;
          if (LOPENBCDRY[L]) continue;
          FP[L] = target(s, f->pser[EFDC_XM_OBC_W], ll, L);
          const int LE = LEC[L];
          if (s.ispb[ll] == 1 || s.ispb[ll] == 2) {
            const double CET = 0.5 * D_LTD2 * G * HRUO[LE] * RCX[LE] * HUc[LE];
            const double TMP = D_LTD2 * std::sqrt(G * HUc[LE]) * DXIU[LE];
            CC[L] = CET * (1. + TMP) / TMP;
            CE[L] = -CET;
            FP[L] = CET * (2. * FP[L] - std::sqrt(G * HUc[LE]) * FUHDYE[LE] * DYIU[LE] / HUc[LE]) / TMP;
          } else {
            const double FP1G = FP[L] / G - HDRY2;
            double CET;
            if (FP1G < BELV[L] || FP1G < BELV[LE]) {
              FP[L] = (BELV[L] + HDRY2) * G;
              CET = 0.;
              LOPENBCDRY[L] = 1;
            } else {
              CET = 0.5 * D_LTD2 * G * HRUO[LE] * RCX[LE] * HUc[LE];
            }
            FP[LE] = FP[LE] + CET * FP[L];
            FP[L] = DE_TI * DXYP[L] * FP[L];
          }
        }
      }
      {  // EAST :77-118
        const Side &s = c->side[EFDC_XM_OBC_E];
        for (int ll = 0; ll < s.n; ++ll) {
          const int L = s.l[ll];
          CC[L] = DELTI * DXYP[L];
          CS[L] = 0.; CW[L] = 0.; CE[L] = 0.; CN[L] = 0.;
          if (LOPENBCDRY[L]) continue;
          FP[L] = target(s, f->pser[EFDC_XM_OBC_E], ll, L);
          if (s.ispb[ll] == 1 || s.ispb[ll] == 2) {
            const double CWT = 0.5 * D_LTD2 * G * HRUO[L] * RCX[L] * HUc[L];
            const double TMP = D_LTD2 * std::sqrt(G * HUc[L]) * DXIU[L];
            CC[L] = CWT * (1. + TMP) / TMP;
            CW[L] = -CWT;
            FP[L] = CWT * (2. * FP[L] + std::sqrt(G * HUc[L]) * FUHDYE[L] * DYIU[L] / HUc[L]) / TMP;
          } else {
            const int LW = LWC[L];
            const double FP1G = FP[L] / G - HDRY2;
            double CWT;
            if (FP1G < BELV[L] || FP1G < BELV[LW]) {
              FP[L] = (BELV[L] + HDRY2) * G;
              CWT = 0.;
              LOPENBCDRY[L] = 1;
            } else {
              CWT = 0.5 * D_LTD2 * G * HRUO[L] * RCX[L] * HUc[L];
            }
            FP[LW] = FP[LW] + CWT * FP[L];
            FP[L] = DE_TI * DXYP[L] * FP[L];
          }
        }
      }
      {  // SOUTH :121-163
        const Side &s = c->side[EFDC_XM_OBC_S];
        for (int ll = 0; ll < s.n; ++ll) {
          const int L = s.l[ll];
          const int LN = LNC[L];
          CC[L] = DELTI * DXYP[L];
          CS[L] = 0.; CW[L] = 0.; CE[L] = 0.; CN[L] = 0.;
          if (LOPENBCDRY[L]) continue;
          FP[L] = target(s, f->pser[EFDC_XM_OBC_S], ll, L);
          if (s.ispb[ll] == 1 || s.ispb[ll] == 2) {
            const double CNT = 0.5 * D_LTD2 * G * HRVO[LN] * RCY[LN] * HVc[LN];
            const double TMP = D_LTD2 * std::sqrt(G * HVc[LN]) * DYIV[LN];
            CC[L] = CNT * (1. + TMP) / TMP;
            CN[L] = -CNT;
            FP[L] = CNT * (2. * FP[L] - std::sqrt(G * HVc[LN]) * FVHDXE[LN] * DXIV[LN] / HVc[LN]) / TMP;
          } else {
            const double FP1G = FP[L] / G - HDRY2;
            double CNT;
            if (FP1G < BELV[L] || FP1G < BELV[LN]) {
              FP[L] = (BELV[L] + HDRY2) * G;
              CNT = 0.;
              LOPENBCDRY[L] = 1;
            } else {
              CNT = 0.5 * D_LTD2 * G * HRVO[LN] * RCY[LN] * HVc[LN];
            }
            FP[LN] = FP[LN] + CNT * FP[L];
            FP[L] = DE_TI * DXYP[L] * FP[L];
          }
        }
      }
      {  // NORTH :166-206
        const Side &s = c->side[EFDC_XM_OBC_N];
        for (int ll = 0; ll < s.n; ++ll) {
          const int L = s.l[ll];
          const int LS = LSC[L];
          CC[L] = DELTI * DXYP[L];
          CS[L] = 0.; CW[L] = 0.; CE[L] = 0.; CN[L] = 0.;
          if (LOPENBCDRY[L]) continue;
          FP[L] = target(s, f->pser[EFDC_XM_OBC_N], ll, L);
          if (s.ispb[ll] == 1 || s.ispb[ll] == 2) {
            const double CST = 0.5 * D_LTD2 * G * HRVO[L] * RCY[L] * HVc[L];
            const double TMP = D_LTD2 * std::sqrt(G * HVc[L]) * DYIV[L];
            CC[L] = CST * (1. + TMP) / TMP;
            CS[L] = -CST;
            FP[L] = CST * (2. * FP[L] + std::sqrt(G * HVc[L]) * FVHDXE[L] * DXIV[L] / HVc[L]) / TMP;
          } else {
            const double FP1G = FP[L] / G - HDRY2;
            double CST;
            if (FP1G < BELV[L] || FP1G < BELV[LS]) {
              FP[L] = (BELV[L] + HDRY2) * G;
              CST = 0.;
              LOPENBCDRY[L] = 1;
            } else {
              CST = 0.5 * D_LTD2 * G * HRVO[L] * RCY[L] * HVc[L];
            }
            FP[LS] = FP[LS] + CST * FP[L];
            FP[L] = DE_TI * DXYP[L] * FP[L];
          }
        }
      }
    }

    // :352-356 implicit sub-grid channel interactions
    if (chans) subchan(c, G, DELT, HDRY, RLAMN, F<const double>{H1P.b}, F<const double>{HP.b},
                       CC, FP);

    // :360-377 minimum diagonal (order-free), FPTMP=FP
    double CCMNM = 1.e+18;
    for (int L = 2; L <= la; ++L) {
      CCMNM = std::min(CCMNM, CC[L]);
      FPTMP[L] = FP[L];
    }
    const double CCMNMI = 1. / CCMNM;
    // :380 SETOPENBC2 (setopenbc2.f90:17-46)
    {
      const Side &w = c->side[EFDC_XM_OBC_W], &e = c->side[EFDC_XM_OBC_E],
                 &s = c->side[EFDC_XM_OBC_S], &n = c->side[EFDC_XM_OBC_N];
      for (int ll = 0; ll < w.n; ++ll)
        if (w.ispb[ll] == 0) CW[LEC[w.l[ll]]] = 0.;
      for (int ll = 0; ll < e.n; ++ll)
        if (e.ispb[ll] == 0) CE[LWC[e.l[ll]]] = 0.;
      for (int ll = 0; ll < s.n; ++ll)
        if (s.ispb[ll] == 0) CS[LNC[s.l[ll]]] = 0.;
      for (int ll = 0; ll < n.n; ++ll)
        if (n.ispb[ll] == 0) CN[LSC[n.l[ll]]] = 0.;
    }
    // :384-399 scale by the minimum diagonal
    for_domains(c, [&](int L) {
      CCS[L] = CS[L] * CCMNMI;
      CCW[L] = CW[L] * CCMNMI;
      CCE[L] = CE[L] * CCMNMI;
      CCN[L] = CN[L] * CCMNMI;
      CCC[L] = CC[L] * CCMNMI;
      FPTMP[L] = FPTMP[L] * CCMNMI;
      CCCI[L] = 1. / CCC[L];
    });

    // :401-405 channel coefficients scaled like the system
    for (int k = 0; k < ch.n; ++k) ch.chh[k] = ch.chh[k] * CCMNMI;

    // :409-410 CONGRAD, or CONGRADC with channels
    int iters = 0;
    double rsq = 0.;
    const int cg =
        congrad(c, P, prm->rsqm, prm->iterm, &iters, &rsq, chans, prm->chan_consistent != 0);
    iters_total += iters;
    last_iters = iters;
    last_rsq = rsq;
    last_ccmnm = CCMNM;
    ++solves;
    if (cg != EFDC_XM_OK) {
      status = cg;
      break;
    }

    // :416-437 face discharges
    for_domains(c, [&](int L) {
      const int LS = LSC[L], LW = LWC[L];
      UHDYE[L] = SUB[L] * (FUHDYE[L] - DELTD2 * HRUO[L] * RCX[L] * HUc[L] * (P[L] - P[LW]));
      VHDXE[L] = SVB[L] * (FVHDXE[L] - DELTD2 * HRVO[L] * RCY[L] * HVc[L] * (P[L] - P[LS]));
    });
    for_domains(c, [&](int L) {
      UHE[L] = UHDYE[L] * DYIU[L];
      VHE[L] = VHDXE[L] * DXIV[L];
    });
    // :440-460 new channel exchange flows
    for (int k = 0; k < ch.n; ++k) {
      const double *P1 = c->p1.data();
      if (ch.iact[k] > 0) {
        const int LHOST = ch.lh[k], LCHNU = ch.lu[k], LCHNV = ch.lv[k];
        if (ch.typ[k] == 1) {
          f->qchanu[k] = ch.cu[k] * ch.qut[k] -
                         RLAMN * ch.cu[k] * ch.cv[k] * (P[LHOST] - P[LCHNU]) -
                         RLAMO * ch.cu[k] * ch.cv[k] * (P1[LHOST] - P1[LCHNU]);
          f->qchanv[k] = 0.;
        }
        if (ch.typ[k] == 2) {
          f->qchanu[k] = 0.;
          f->qchanv[k] = ch.cu[k] * ch.qvt[k] -
                         RLAMN * ch.cu[k] * ch.cv[k] * (P[LHOST] - P[LCHNV]) -
                         RLAMO * ch.cu[k] * ch.cv[k] * (P1[LHOST] - P1[LCHNV]);
        }
      } else {
        f->qchanv[k] = 0.;
        f->qchanvn[k] = 0.;
        f->qchanu[k] = 0.;
        f->qchanun[k] = 0.;
      }
    }
    // :466-486 continuity
    if (!tl3) {
      for_domains(c, [&](int L) {
        const int LE = LEC[L], LN = LNC[L];
        HP[L] = H1P[L] + DELTD2 * DXYIP[L] *
                             (2. * QSUME[L] - (UHDYE[LE] + UHDY1E[LE] - UHDYE[L] - UHDY1E[L] +
                                               VHDXE[LN] + VHDX1E[LN] - VHDXE[L] - VHDX1E[L]));
      });
    } else {  // calpuv9c.f90:500-525: from level n-1 (ISTL_ = 3) or n (ISTL_ = 2)
      const F<double> HB = (ISTL == 3) ? H2P : H1P, UB = (ISTL == 3) ? U2 : U1,
                      VB = (ISTL == 3) ? V2 : V1;
      for_domains(c, [&](int L) {
        const int LE = LEC[L], LN = LNC[L];
        HP[L] = HB[L] + DELT * DXYIP[L] *
                            (QSUME[L] - 0.5 * (UHDYE[LE] + UB[LE] - UHDYE[L] - UB[L] +
                                               VHDXE[LN] + VB[LN] - VHDXE[L] - VB[L]));
      });
    }
    // :489-535 open boundaries
    for (int L : c->lobcs) {
      HP[L] = GI * P[L] - BELV[L];
      if (ISDRY > 0) {
        if ((LOPENBCDRY[L] || (H1P[L] < 0.9 * HDRY && HP[L] < H1P[L]) || HP[L] < 0.) &&
            ISCDRY[L] == 0) {
          if (HP[L] <= 0. && LOPENBCDRY[L]) {
            HP[L] = 0.2 * HDRY;
          } else {
            HP[L] = std::min(std::max(H1P[L], 0.1 * HDRY), 0.9 * HDRY);
          }
          ISCDRY[L] = 1;
          const int LE = LEC[L], LN = LNC[L];
          SUB[L] = 0.; SVB[L] = 0.; SUB[LE] = 0.; SVB[LN] = 0.;
          SBX[L] = 0.; SBY[L] = 0.; SBX[LE] = 0.; SBY[LN] = 0.;
          UHDYE[L] = 0.; UHDYE[LE] = 0.; VHDXE[L] = 0.; VHDXE[LN] = 0.;
          LOPENBCDRY[L] = 1;
          CC[L] = DELTI * DXYP[L];
          P[L] = (HP[L] + BELV[L]) * G;
          FP1[L] = DELTI * DXYP[L] * P[L];
        }
      }
    }
    // :538-556 channel exchanges
    for (int k = 0; k < ch.n; ++k) {
      if (ch.iact[k] > 0) {
        const int LHOST = ch.lh[k], LCHNU = ch.lu[k], LCHNV = ch.lv[k];
        if (ch.typ[k] == 1) {
          const double TMPVAL = DELT * (RLAMN * f->qchanu[k] + RLAMO * ch.qut[k]);
          HP[LHOST] = HP[LHOST] + TMPVAL * DXYIP[LHOST];
          HP[LCHNU] = HP[LCHNU] - TMPVAL * DXYIP[LCHNU];
        }
        if (ch.typ[k] == 2) {
          const double TMPVAL = DELT * (RLAMN * f->qchanv[k] + RLAMO * ch.qvt[k]);
          HP[LHOST] = HP[LHOST] + TMPVAL * DXYIP[LHOST];
          HP[LCHNV] = HP[LCHNV] - TMPVAL * DXYIP[LCHNV];
        }
      }
    }
    // :557-571 intermediate P update
    if (ISDRY > 0) for_domains(c, [&](int L) { P[L] = G * (HP[L] + BELV[L]); });

    // :574-603 legacy drying check, ISDRY 1..97 (serial in the reference)
    if (ISDRY > 0 && ISDRY < 98) {
      int ICORDRY = 0;
      const double HDRY90 = 0.9 * HDRY, HDRY10 = 0.1 * HDRY;
      for (int L = 2; L <= la; ++L) {
        const int LE = LEC[L], LN = LNC[L];
        bool dry = HP[L] <= HDRY;
        if (tl3) {  // calpuv9c.f90:628-662: only a cell below HDRY that is not rising fast
          const double HPPMC = (ISTL == 3) ? H2P[L] : H1P[L];
          dry = HP[L] < HDRY && (HP[L] < HDRY90 || HPPMC < HDRY) && HP[L] < (HPPMC + HDRY10);
        }
        if (dry) {
          if (ISCDRY[L] == 0) {
            ISCDRY[L] = 1;
            ICORDRY = 1;
          }
          SUB[L] = 0.; SVB[L] = 0.; SUB[LE] = 0.; SVB[LN] = 0.;
          SBX[L] = 0.; SBY[L] = 0.; SBX[LE] = 0.; SBY[LN] = 0.;
        }
      }
      if (ICORDRY == 1) {
        ++NCORDRY;
        if (NCORDRY < max_sweeps) continue;
        status = EFDC_XM_WETDRY_MAXSWEEP;
        break;
      }
    }

    // :606-734 ISDRY=99 drying/rewetting.  Restated with the 1-thread (serial
    // L-order) semantics: the reference's OMP split can race on faces shared
    // by two domains; the serial order is its thread-count-1 result.
    if (ISDRY == 99) {
      const double HDRY2 = 2. * HDRY;
      const double HDRY90 = 0.9 * HDRY;
      int ICORDRY = 0;
      for (int L = 2; L <= la; ++L) {
        const int LW = LWC[L], LE = LEC[L], LS = LSC[L], LN = LNC[L];
        if (HP[L] <= HDRY) {
          const double SUBW = SUB[L], SUBE = SUB[LE], SVBS = SVB[L], SVBN = SVB[LN];
          // HPPMC: H2P in CALPUV9C(3) (calpuv9c.f90:679-686), else H1P
          const double HPPMC = (ISTL == 3) ? H2P[L] : H1P[L];
          const double DHPDT = (HP[L] - HPPMC);
          if (DHPDT > 0.0) {
            SUB[L] = 0.0; SUB[LE] = 0.0; SVB[L] = 0.0; SVB[LN] = 0.0;
            SBX[L] = 0.0; SBX[LE] = 0.0; SBY[L] = 0.0; SBY[LN] = 0.0;
            const double DHPDT2 = (HDRY - HPPMC) * 0.01;
            if (DHPDT > DHPDT2) {
              if (SUBO[L] > 0.5)
                if (UHDYE[L] > 0.0 && HP[LW] > HDRY2) { SUB[L] = SUBO[L]; SBX[L] = SBXO[L]; }
              if (SUBO[LE] > 0.5)
                if (UHDYE[LE] < 0.0 && HP[LE] > HDRY2) { SUB[LE] = SUBO[LE]; SBX[LE] = SBXO[LE]; }
              if (SVBO[L] > 0.5)
                if (VHDXE[L] > 0.0 && HP[LS] > HDRY2) { SVB[L] = SVBO[L]; SBY[L] = SBYO[L]; }
              if (SVBO[LN] > 0.5)
                if (VHDXE[LN] < 0.0 && HP[LN] > HDRY2) { SVB[LN] = SVBO[LN]; SBY[LN] = SBYO[LN]; }
              const double RDRY = SUB[L] + SUB[LE] + SVB[L] + SVB[LN];
              ISCDRY[L] = (RDRY < 0.5) ? 1 : 0;
              if (std::fabs(SUB[L] - SUBW) > 0.5) ICORDRY = 1;
              else if (std::fabs(SUB[LE] - SUBE) > 0.5) ICORDRY = 1;
              else if (std::fabs(SVB[L] - SVBS) > 0.5) ICORDRY = 1;
              else if (std::fabs(SVB[LN] - SVBN) > 0.5) ICORDRY = 1;
            } else {
              if (ISCDRY[L] == 0) {
                ISCDRY[L] = 1;
                ICORDRY = 1;
              }
            }
          } else if (HP[L] < HDRY90 || HPPMC < HDRY) {
            SUB[L] = 0.0; SUB[LE] = 0.0; SVB[L] = 0.0; SVB[LN] = 0.0;
            SBX[L] = 0.0; SBX[LE] = 0.0; SBY[L] = 0.0; SBY[LN] = 0.0;
            if (ISCDRY[L] == 0) {
              ISCDRY[L] = 1;
              ICORDRY = 1;
            }
          }
        }
      }
      if (ICORDRY > 0) {
        ++NCORDRY;
        if (NCORDRY < max_sweeps) continue;
        status = EFDC_XM_WETDRY_MAXSWEEP;
        break;
      }
    }
    break;
  }

  st->iters_last = last_iters;
  st->iters_total = iters_total;
  st->solves = solves;
  st->rsq_last = last_rsq;
  st->ccmnm_last = last_ccmnm;
  if (status == EFDC_XM_CG_MAXITER || status == EFDC_XM_NONFINITE ||
      status == EFDC_XM_WETDRY_MAXSWEEP) {
    st->status = status;
    return status;
  }

  // ---- final domain loop (:829-969), 1-thread order: volume wasting for all
  // cells first, then the depth updates that read neighbour HP.
  int n_wasted = 0;
  if (ISDRY > 0 && NDRYSTP < 0) {  // :838-889
    const int NTMP = std::abs(NDRYSTP);
    for (int L = 2; L <= la; ++L) {
      if (HP[L] >= HDRY) {
        const int LW = LWC[L], LE = LEC[L], LS = LSC[L], LN = LNC[L];
        const double RDRY = SUB[L] + SUB[LE] + SVB[L] + SVB[LN];
        if (RDRY > 0.5) {
          NATDRY[L] = 0;
        } else {
          NATDRY[L] = NATDRY[L] + 1;
          if (NATDRY[L] > NTMP) {
            double RVAL = 0.0;
            if (SUBO[LE] > 0.5 && BELV[LE] < BELV[L]) RVAL = RVAL + 1.;
            if (SUBO[L] > 0.5 && BELV[LW] < BELV[L]) RVAL = RVAL + 1.;
            if (SVBO[LN] > 0.5 && BELV[LN] < BELV[L]) RVAL = RVAL + 1.;
            if (SVBO[L] > 0.5 && BELV[LS] < BELV[L]) RVAL = RVAL + 1.;
            if (RVAL > 0. || HP[L] < HDRY * 2.) {
              const double HOLDTMP = HP[L];
              H1P[L] = HP[L];
              HP[L] = 0.90 * HDRY;
              NATDRY[L] = 0;
              // CALPUV9C adds to the QDWASTE it zeroed at entry (calpuv9c.f90:919)
              QDWASTE[L] = tl3 ? QDWASTE[L] + DELTI * DXYP[L] * (HOLDTMP - HP[L])
                               : DELTI * DXYP[L] * (HOLDTMP - HP[L]);
              VDWASTE[L] = VDWASTE[L] + DXYP[L] * (HOLDTMP - HP[L]);
              nnatdry_flag[L] = 1;
              ++n_wasted;
            }
          }
        }
      }
    }
  }
  for_domains(c, [&](int L) {
    if (ISDRY == 0) P[L] = G * (HP[L] + BELV[L]);  // :893-897
  });
  for_domains(c, [&](int L) {  // :898-906
    const int LS = LSC[L], LW = LWC[L];
    HU[L] = (DXYP[L] * HP[L] + DXYP[LW] * HP[LW]) * FSGZU[L];
    HV[L] = (DXYP[L] * HP[L] + DXYP[LS] * HP[LS]) * FSGZV[L];
  });
  for_domains(c, [&](int L) {
    HPI[L] = 1. / HP[L];
    HUI[L] = 1. / HU[L];
    HVI[L] = 1. / HV[L];
  });
  if (ISDRY > 0) {  // :910-931
    for_domains(c, [&](int L) {
      LMASKDRY[L] = 1;
      if (HP[L] < HDRY) {
        const int LE = LEC[L], LN = LNC[L];
        int IUW = 0, IUE = 0, IVS = 0, IVN = 0;
        if (SUB1[L] < 0.5 && SUB[L] < 0.5) IUE = 1;
        if (SUB1[LE] < 0.5 && SUB[LE] < 0.5) IUW = 1;
        if (SVB1[L] < 0.5 && SVB[L] < 0.5) IVS = 1;
        if (SVB1[LN] < 0.5 && SVB[LN] < 0.5) IVN = 1;
        if (IUW + IUE + IVS + IVN == 4) LMASKDRY[L] = 0;
      }
    });
  }
  // :1003-1025 wasted cells: H1P reset, QDWASTE kept only with ISBAL>0
  // (CALPUV9C resets H1P only, calpuv9c.f90:1047-1058)
  if (n_wasted > 0) {
    for (int L = 2; L <= la; ++L)
      if (nnatdry_flag[L]) {
        H1P[L] = 0.90 * HDRY;
        if (prm->isbal == 0 && !tl3) QDWASTE[L] = 0.0;
      }
  }
  // NEGDEP check (negdep.f90:34-45)
  int nneg = 0;
  for (int L = 2; L <= la; ++L)
    if (HP[L] <= 0.) ++nneg;
  // wet/dry cell lists (:1061-1080)
  int lawet = 0, ladry = 0;
  if (ISDRY == 0) {
    lawet = la - 1;
    if (f->lwet)
      for (int L = 2; L <= la; ++L) f->lwet[L - 2] = L;
  } else {
    for (int L = 2; L <= la; ++L) {
      if (LMASKDRY[L]) {
        if (f->lwet) f->lwet[lawet] = L;
        ++lawet;
      } else if (OLDMASK[L] || prm->n < prm->ntstbc + 1) {
        if (f->ldry) f->ldry[ladry] = L;
        ++ladry;
      }
    }
  }
  st->lawet = lawet;
  st->ladry = ladry;
  st->n_negdep = nneg;
  st->n_wasted = n_wasted;
  for (int L = 2; L <= la; ++L)
    if (!std::isfinite(P[L])) {
      status = EFDC_XM_NONFINITE;
      break;
    }
  if (status == EFDC_XM_OK && nneg > 0) status = EFDC_XM_NEG_DEPTH;
  // optional diagnostics of the last sweep
  if (f->ccc) for (int L = 1; L <= lc; ++L) f->ccc[L - 1] = CCC[L];
  if (f->ccs) for (int L = 1; L <= lc; ++L) f->ccs[L - 1] = CCS[L];
  if (f->ccw) for (int L = 1; L <= lc; ++L) f->ccw[L - 1] = CCW[L];
  if (f->cce) for (int L = 1; L <= lc; ++L) f->cce[L - 1] = CCE[L];
  if (f->ccn) for (int L = 1; L <= lc; ++L) f->ccn[L - 1] = CCN[L];
  if (f->fptmp) for (int L = 1; L <= lc; ++L) f->fptmp[L - 1] = FPTMP[L];
  st->status = status;
  return status;
}

int oracle_set_layers(oracle_ctx *c, const efdc_xm_layers *ly) {
  if (!ly || ly->kc < 1 || ly->kc > 64 || ly->ld < c->lc || !ly->dzc || !ly->zz)
    return EFDC_XM_BAD_ARGUMENT;
  const size_t ldl = size_t(c->lc) + 2;
  c->kc = ly->kc;
  c->dzc.assign(ldl * ly->kc, 0.0);
  c->zz.assign(ldl * ly->kc, 0.0);
  for (int k = 0; k < ly->kc; ++k)
    for (int L = 1; L <= c->lc; ++L) {
      c->dzc[k * ldl + L] = ly->dzc[size_t(k) * ly->ld + (L - 1)];
      c->zz[k * ldl + L] = ly->zz[size_t(k) * ly->ld + (L - 1)];
    }
  c->bi1.assign(ldl, 0.0);
  c->bi2.assign(ldl, 0.0);
  c->be.assign(ldl, 0.0);
  return EFDC_XM_OK;
}

int oracle_set_channels(oracle_ctx *c, const efdc_xm_channels *in) {
  Channels &ch = c->ch;
  ch = Channels{};
  if (!in || in->n <= 0) return EFDC_XM_OK;
  const int n = in->n;
  if (!in->type || !in->lhost || !in->lu || !in->lv || !in->chanlen || !in->chanfric ||
      !in->dxp || !in->dyp)
    return EFDC_XM_BAD_ARGUMENT;
  ch.n = n;
  ch.typ.assign(in->type, in->type + n);
  ch.lh.assign(in->lhost, in->lhost + n);
  ch.lu.assign(in->lu, in->lu + n);
  ch.lv.assign(in->lv, in->lv + n);
  ch.len.assign(in->chanlen, in->chanlen + n);
  ch.fric.assign(in->chanfric, in->chanfric + n);
  copy1(ch.dxp, in->dxp, c->lc);
  copy1(ch.dyp, in->dyp, c->lc);
  for (auto *v : {&ch.cu, &ch.cv, &ch.chh, &ch.qut, &ch.qvt}) v->assign(n, 0.0);
  ch.iact.assign(n, 0);
  c->p1.assign(size_t(c->lc) + 2, 0.0);
  return EFDC_XM_OK;
}

int oracle_set_bed(oracle_ctx *c, const efdc_xm_bed *b) {
  if (!c || !b || !b->zbr || !b->stbxo || !b->stbyo || !b->dxp || !b->dyp || !b->dzc1 ||
      !b->sgzu1 || !b->sgzv1 || b->kc < 1)
    return EFDC_XM_BAD_ARGUMENT;
  const int lc = c->lc, la = c->la;
  copy1(c->zbr, b->zbr, lc);
  copy1(c->stbxo, b->stbxo, lc);  // STBXO(L)=STBX(L) (caltbxy.f90:108-111)
  copy1(c->stbyo, b->stbyo, lc);
  std::vector<double> dxp, dyp, dzc1, sgzu1, sgzv1;
  copy1(dxp, b->dxp, lc);
  copy1(dyp, b->dyp, lc);
  copy1(dzc1, b->dzc1, lc);
  copy1(sgzu1, b->sgzu1, lc);
  copy1(sgzv1, b->sgzv1, lc);
  c->zbratu.assign(size_t(lc) + 2, 0.);
  c->zbratv.assign(size_t(lc) + 2, 0.);
  c->sgzuu.assign(size_t(lc) + 2, 0.);
  c->sgzvv.assign(size_t(lc) + 2, 0.);
  for (int L = 2; L <= la; ++L) {  // caltbxy.f90:81-90 (layer 1: KSZU = KSZV = 1)
    const int LW = c->lwc[L], LS = c->lsc[L];
    c->zbratu[L] = 0.5 * (dxp[LW] * c->zbr[LW] + dxp[L] * c->zbr[L]) * c->dxiu[L];
    c->zbratv[L] = 0.5 * (dyp[LS] * c->zbr[LS] + dyp[L] * c->zbr[L]) * c->dyiv[L];
    c->sgzuu[L] = 0.5 * std::max(dzc1[L], sgzu1[L]);
    c->sgzvv[L] = 0.5 * std::max(dzc1[L], sgzv1[L]);
  }
  c->stbx.assign(size_t(lc) + 2, 0.);  // STBX(L)=0. (:112-116)
  c->stby.assign(size_t(lc) + 2, 0.);
  c->bed_kc = b->kc;
  c->avcon = b->avcon;
  c->vismud = b->vismud;
  c->visfac = 0.0258 * std::pow(b->coeftsbl, 2. / 7.);  // :210-211
  c->bed = true;
  return EFDC_XM_OK;
}

int oracle_bottom_stress(oracle_ctx *c, const efdc_xm_drag_params *p, const efdc_xm_fields *st,
                         efdc_xm_drag_fields *f) {
  if (!c || !p || !st || !f || !c->bed || !st->hu || !st->hv || !f->ub || !f->vb || !f->vu ||
      !f->uv || !f->h1u || !f->h1v || !f->tbx || !f->tby || !(p->delt > 0) ||
      (p->isdry > 0 && !st->lmaskdry))
    return EFDC_XM_BAD_ARGUMENT;
  const int la = c->la;
  const F<const double> HU{st->hu}, HV{st->hv}, U{f->ub}, V{f->vb}, VU{f->vu}, UV{f->uv},
      H1U{f->h1u}, H1V{f->h1v};
  F<double> TBX{f->tbx}, TBY{f->tby};
  const double DELT = p->delt;
  const double CDLIMIT = 0.5;        // ISITB = 0 (caltbxy.f90:172-180)
  const double VISEXP = 2. / 7.;     // :210
  const double VISFAC = c->visfac;
  const double AVCON = c->avcon;
  double *STBX = c->stbx.data(), *STBY = c->stby.data();
  const double *STBXO = c->stbxo.data(), *STBYO = c->stbyo.data(), *ZBR = c->zbr.data();
  auto wet = [&](int L) { return p->isdry == 0 || st->lmaskdry[L - 1] != 0; };
  // :213-229 cells of LDRY (calpuv2c.f90:1061-1080): TBX, TBY of their faces to zero
  if (p->isdry > 0)
    for (int L = 2; L <= la; ++L) {
      if (wet(L) || !(c->oldmask[L] || p->n < p->ntstbc + 1)) continue;
      TBX[L] = 0.;
      TBY[L] = 0.;
      TBX[c->lec[L]] = 0.;
      TBY[c->lnc[L]] = 0.;
    }
  for (int L = 2; L <= la; ++L) {  // :476-539 over LWET
    if (!wet(L)) continue;
    if (ZBR[L] <= 1.E-6) {  // :480-502 smooth (viscous) drag, ISMUD = 0
      const double UMAGTMP = std::sqrt(U[L] * U[L] + VU[L] * VU[L] + 1.E-12);
      const double VMAGTMP = std::sqrt(UV[L] * UV[L] + V[L] * V[L] + 1.E-12);
      const double CDMAXU = CDLIMIT * STBXO[L] * HU[L] / (DELT * UMAGTMP);
      const double CDMAXV = CDLIMIT * STBYO[L] * HV[L] / (DELT * VMAGTMP);
      const double HUI = 1. / HU[L], HVI = 1. / HV[L];
      double VISDHU = 0.0, VISDHV = 0.0;
      if (UMAGTMP > 0.0) VISDHU = (c->vismud * HUI / UMAGTMP) * VISEXP;
      if (VMAGTMP > 0.0) VISDHV = (c->vismud * HVI / VMAGTMP) * VISEXP;
      STBX[L] = VISFAC * AVCON * STBXO[L] * VISDHU;
      STBY[L] = VISFAC * AVCON * STBYO[L] * VISDHV;
      STBX[L] = std::min(CDMAXU, STBX[L]);
      STBY[L] = std::min(CDMAXV, STBY[L]);
    } else {  // :504-537 rough (log-law) drag
      const double UMAGTMP = std::sqrt(VU[L] * VU[L] + U[L] * U[L] + 1.E-12);
      const double VMAGTMP = std::sqrt(UV[L] * UV[L] + V[L] * V[L] + 1.E-12);
      const double CDMAXU = CDLIMIT * STBXO[L] * HU[L] / (DELT * UMAGTMP);
      const double CDMAXV = CDLIMIT * STBYO[L] * HV[L] / (DELT * VMAGTMP);
      const double HURTMP = std::max(c->zbratu[L], H1U[L]);
      const double HVRTMP = std::max(c->zbratv[L], H1V[L]);
      if (c->bed_kc == 1) {  // KSZ(L) == KC
        double HUDZBR = 0.5 * HURTMP / c->zbratu[L];
        HUDZBR = std::max(HUDZBR, 7.5);
        double HVDZBR = 0.5 * HVRTMP / c->zbratv[L];
        HVDZBR = std::max(HVDZBR, 7.5);
        const double lu = std::log(HUDZBR) - 1., lv = std::log(HVDZBR) - 1.;
        STBX[L] = STBXO[L] * .16 / (lu * lu);
        STBY[L] = STBYO[L] * .16 / (lv * lv);
      } else {
        double DZHUDZBR = 1. + c->sgzuu[L] * HURTMP / c->zbratu[L];
        double DZHVDZBR = 1. + c->sgzvv[L] * HVRTMP / c->zbratv[L];
        DZHUDZBR = std::max(DZHUDZBR, 7.5);
        DZHVDZBR = std::max(DZHVDZBR, 7.5);
        const double lu = std::log(DZHUDZBR), lv = std::log(DZHVDZBR);
        STBX[L] = AVCON * STBXO[L] * .16 / (lu * lu);
        STBY[L] = AVCON * STBYO[L] * .16 / (lv * lv);
      }
      STBX[L] = std::min(CDMAXU, STBX[L]);
      STBY[L] = std::min(CDMAXV, STBY[L]);
    }
  }
  for (int L = 2; L <= la; ++L) {  // hdmt2t.f90:670-684 over LWET
    if (!wet(L)) continue;
    const double USGZ = U[L], VSGZ = V[L];
    TBX[L] = (p->avcon1 * (1. / HU[L]) + STBX[L] * std::sqrt(VU[L] * VU[L] + USGZ * USGZ)) * USGZ;
    TBY[L] = (p->avcon1 * (1. / HV[L]) + STBY[L] * std::sqrt(UV[L] * UV[L] + VSGZ * VSGZ)) * VSGZ;
  }
  for (int L = 1; L <= c->lc; ++L) {
    if (f->stbx) f->stbx[L - 1] = STBX[L];
    if (f->stby) f->stby[L - 1] = STBY[L];
  }
  return EFDC_XM_OK;
}

int oracle_set_momentum(oracle_ctx *c, const efdc_xm_momentum *mo) {
  const int lc = c->lc;
  if (!mo || mo->kc < 1 || mo->kc > 64 || mo->ld < lc || !mo->fcorc || !mo->dydi ||
      !mo->dxdj || !mo->scax || !mo->scay || !mo->saax || !mo->saay || !mo->sgzu ||
      !mo->sgzv || !mo->fsgzu || !mo->fsgzv || !mo->lnwc || !mo->lsec || mo->nbcs < 0)
    return EFDC_XM_BAD_ARGUMENT;
  const int kc = mo->kc, n1 = lc + 2;
  c->mom = true;
  c->mkc = kc;
  c->mld = mo->ld;
  copy1(c->fcorc, mo->fcorc, lc);
  copy1(c->dydi, mo->dydi, lc);
  copy1(c->dxdj, mo->dxdj, lc);
  copy1(c->scax, mo->scax, lc);
  copy1(c->scay, mo->scay, lc);
  copy1(c->saax, mo->saax, lc);
  copy1(c->saay, mo->saay, lc);
  copy1(c->stcuv, mo->stcuv, lc);
  if (!mo->stcuv) c->stcuv.clear();
  copy1(c->sdx, mo->sdx, lc);
  copy1(c->sdy, mo->sdy, lc);
  copy1(c->lhdmf, mo->lhdmf, lc);
  copy1(c->lnwc, mo->lnwc, lc);
  copy1(c->lsec, mo->lsec, lc);
  for (auto *v : {&c->msgzu, &c->msgzv, &c->mfsgzu, &c->mfsgzv}) v->assign(size_t(kc) * n1, 0.);
  for (int k = 0; k < kc; ++k)
    for (int L = 1; L <= lc; ++L) {
      const size_t i = size_t(k) * n1 + L, j = size_t(k) * mo->ld + L - 1;
      c->msgzu[i] = mo->sgzu[j];
      c->msgzv[i] = mo->sgzv[j];
      c->mfsgzu[i] = mo->fsgzu[j];
      c->mfsgzv[i] = mo->fsgzv[j];
    }
  c->lbcs.assign(mo->lbcs, mo->lbcs + mo->nbcs);
  c->lberc.assign(mo->lberc, mo->lberc + mo->nbcs);
  c->lbnrc.assign(mo->lbnrc, mo->lbnrc + mo->nbcs);
  for (auto *v : {&c->fuhu, &c->fvhu, &c->fvhv, &c->fuhv, &c->cac, &c->fcax, &c->fcay, &c->fx,
                  &c->fy})
    v->assign(size_t(kc) * n1, 0.);
  c->mwet_prev.assign(n1, 0);
  return EFDC_XM_OK;
}

// CALEXP2T (calexp2t.f90:129-956) for IS2LMC = 0 and the options of
// efdc_xm_explicit_batch, serially in the reference's statement order.  The
// layer arrays are the context's, kept between calls; the caller's FCAXE,
// FCAYE, FXE, FYE are in/out like the module arrays.
int oracle_explicit(oracle_ctx *c, const efdc_xm_explicit_params *p,
                    efdc_xm_explicit_fields *f) {
  if (!c->mom || !p || !f || !f->u || !f->v || !f->uhdy || !f->vhdx || !f->hp || !f->fcaxe ||
      !f->fcaye || !f->fxe || !f->fye)
    return EFDC_XM_BAD_ARGUMENT;
  if (p->ishdmf >= 1 && (c->sdx.empty() || !f->fmdux || !f->fmduy || !f->fmdvx || !f->fmdvy ||
                         c->lhdmf.empty()))
    return EFDC_XM_BAD_ARGUMENT;
  const int la = c->la, lc = c->lc, kc = c->mkc, n1 = lc + 2;
  auto K_ = [&](std::vector<double> &v, int k) { return F<double>{v.data() + size_t(k) * n1 + 1}; };
  std::vector<int> wet(n1, 0);
  for (int L = 2; L <= la; ++L) wet[L] = f->wet ? (f->wet[L - 1] != 0) : 1;
  std::vector<int> lwet;  // LWET in L order
  for (int L = 2; L <= la; ++L)
    if (wet[L]) lwet.push_back(L);
  F<double> FCAXE{f->fcaxe}, FCAYE{f->fcaye}, FXE{f->fxe}, FYE{f->fye}, HP{const_cast<double *>(f->hp)};
  F<double> DXYP{c->dxyp.data() + 1}, FCORC{c->fcorc.data() + 1}, DYDI{c->dydi.data() + 1},
      DXDJ{c->dxdj.data() + 1}, SCAX{c->scax.data() + 1}, SCAY{c->scay.data() + 1},
      SAAX{c->saax.data() + 1}, SAAY{c->saay.data() + 1};
  F<int> LEC{c->lec.data() + 1}, LWC{c->lwc.data() + 1}, LNC{c->lnc.data() + 1},
      LSC{c->lsc.data() + 1}, LNWC{c->lnwc.data() + 1}, LSEC{c->lsec.data() + 1};
  // the caller's layer arrays (leading dimension LCM), layer k (0-based) of element L
  const long cld = c->mld;
  auto in = [&](const double *a, int k, int L) { return a ? a[size_t(k) * cld + L - 1] : 0.0; };
  const double SNLT = p->snlt;
  // :131-175 newly dry cells (wet at the previous call, not now): zero the
  // sums and every layer array
  for (int L = 2; L <= la; ++L)
    if (c->mwet_prev[L] && !wet[L]) {
      FCAXE[L] = 0.;
      FCAYE[L] = 0.;
      FXE[L] = 0.;
      FYE[L] = 0.;
      for (int k = 0; k < kc; ++k)
        for (auto *v : {&c->fuhu, &c->fvhu, &c->fvhv, &c->fuhv, &c->cac, &c->fcax, &c->fcay,
                        &c->fx, &c->fy})
          K_(*v, k)[L] = 0.;
    }
  c->mwet_prev = wet;
  // :187-197
  for (int L : lwet) {
    FCAXE[L] = 0.;
    FCAYE[L] = 0.;
    FXE[L] = 0.;
    FYE[L] = 0.;
  }
  // :205-237 upwind momentum fluxes
  for (int k = 0; k < kc; ++k) {
    F<double> FUHU = K_(c->fuhu, k), FVHU = K_(c->fvhu, k), FVHV = K_(c->fvhv, k),
              FUHV = K_(c->fuhv, k);
    for (int L : lwet) {
      const int LE = LEC[L], LN = LNC[L], LS = LSC[L], LW = LWC[L];
      const double UHB = 0.5 * (in(f->uhdy, k, L) + in(f->uhdy, k, LE));
      const double VHC = 0.5 * (in(f->vhdx, k, L) + in(f->vhdx, k, LW));
      FUHU[L] = std::max(UHB, 0.) * in(f->u, k, L) + std::min(UHB, 0.) * in(f->u, k, LE);
      FVHU[L] = std::max(VHC, 0.) * in(f->u, k, LS) + std::min(VHC, 0.) * in(f->u, k, L);
      const double VHB = 0.5 * (in(f->vhdx, k, L) + in(f->vhdx, k, LN));
      const double UHC = 0.5 * (in(f->uhdy, k, L) + in(f->uhdy, k, LS));
      FVHV[L] = std::max(VHB, 0.) * in(f->v, k, L) + std::min(VHB, 0.) * in(f->v, k, LN);
      FUHV[L] = std::max(UHC, 0.) * in(f->v, k, LW) + std::min(UHC, 0.) * in(f->v, k, L);
    }
  }
  // :460-472 triangular cells
  if (!c->stcuv.empty())
    for (int k = 0; k < kc; ++k)
      for (int L : lwet) {
        K_(c->fuhu, k)[L] = c->stcuv[L] * K_(c->fuhu, k)[L];
        K_(c->fvhv, k)[L] = c->stcuv[L] * K_(c->fvhv, k)[L];
      }
  // :481-535 Coriolis-curvature coefficients and their sum
  double CACSUMT = 0.;
  if (p->iscurvature) {
    double sum = 0.;
    for (int k = 0; k < kc; ++k) {
      F<double> CAC = K_(c->cac, k);
      for (int L : lwet) {
        const int LE = LEC[L], LN = LNC[L];
        CAC[L] = (FCORC[L] * DXYP[L] + 0.5 * SNLT * (in(f->v, k, LN) + in(f->v, k, L)) * DYDI[L] -
                  0.5 * SNLT * (in(f->u, k, LE) + in(f->u, k, L)) * DXDJ[L]) *
                 HP[L];
        sum = sum + CAC[L];
      }
    }
    CACSUMT = std::fabs(sum);
    if (CACSUMT < 1.E-7)
      for (int k = 0; k < kc; ++k)
        for (int L : lwet) {
          K_(c->fcax, k)[L] = 0.;
          K_(c->fcay, k)[L] = 0.;
        }
  }
  // :545-562
  if (CACSUMT > 1.E-7)
    for (int k = 0; k < kc; ++k) {
      F<double> CAC = K_(c->cac, k), FCAX = K_(c->fcax, k), FCAY = K_(c->fcay, k);
      for (int L : lwet) {
        const int LE = LEC[L], LN = LNC[L], LS = LSC[L], LW = LWC[L], LNW = LNWC[L],
                  LSE = LSEC[L];
        FCAX[L] = 0.25 * SCAX[L] *
                  (CAC[L] * (in(f->v, k, LN) + in(f->v, k, L)) +
                   CAC[LW] * (in(f->v, k, LNW) + in(f->v, k, LW)));
        FCAY[L] = 0.25 * SCAY[L] *
                  (CAC[L] * (in(f->u, k, LE) + in(f->u, k, L)) +
                   CAC[LS] * (in(f->u, k, LSE) + in(f->u, k, LS)));
      }
    }
  // :605-645 type-2 open boundaries
  for (int s = 0; s < 4; ++s) {
    const Side &sd = c->side[s];
    for (int ll = 0; ll < sd.n; ++ll) {
      if (sd.ispb[ll] != 2) continue;
      const int LB = sd.l[ll];
      for (int k = 0; k < kc; ++k) {
        F<double> CAC = K_(c->cac, k), FCAX = K_(c->fcax, k), FCAY = K_(c->fcay, k);
        if (s == 0) {  // W: the cell after the boundary cell in L order (:607-614)
          const int L = LB + 1, LN = LNC[L];
          FCAX[L] = 0.5 * SCAX[L] * CAC[L] * (in(f->v, k, LN) + in(f->v, k, L));
        } else if (s == 1) {  // E (:617-624)
          const int L = LB, LNW = LNWC[L], LW = LWC[L];
          FCAX[L] = 0.5 * SCAX[L] * CAC[LW] * (in(f->v, k, LNW) + in(f->v, k, LW));
        } else if (s == 2) {  // S: the boundary cell's north neighbour (:627-633)
          const int L = LNC[LB], LE = LEC[L];
          FCAY[L] = 0.5 * SCAY[L] * CAC[L] * (in(f->u, k, LE) + in(f->u, k, L));
        } else {  // N (:636-643)
          const int L = LB, LS = LSC[L], LSE = LSEC[L];
          FCAY[L] = 0.5 * SCAY[L] * CAC[LS] * (in(f->u, k, LSE) + in(f->u, k, LS));
        }
      }
    }
  }
  // :648-662 layer forcings with the gross momentum
  for (int k = 0; k < kc; ++k) {
    F<double> FUHU = K_(c->fuhu, k), FVHU = K_(c->fvhu, k), FVHV = K_(c->fvhv, k),
              FUHV = K_(c->fuhv, k), FX = K_(c->fx, k), FY = K_(c->fy, k);
    F<double> FSGZU{c->mfsgzu.data() + size_t(k) * n1 + 1},
        FSGZV{c->mfsgzv.data() + size_t(k) * n1 + 1};
    for (int L : lwet) {
      const int LE = LEC[L], LN = LNC[L], LS = LSC[L], LW = LWC[L];
      FX[L] = FSGZU[L] * (FUHU[L] - FUHU[LW] + FVHU[LN] - FVHU[L]) + in(f->fuhj, k, L);
      FY[L] = FSGZV[L] * (FVHV[L] - FVHV[LS] + FUHV[LE] - FUHV[L]) + in(f->fvhj, k, L);
    }
  }
  // :664-689 flow-boundary edges
  for (size_t ll = 0; ll < c->lbcs.size(); ++ll)
    for (int k = 0; k < kc; ++k) {
      F<double> FX = K_(c->fx, k), FY = K_(c->fy, k);
      int L = c->lbcs[ll];
      FX[L] = SAAX[L] * FX[L] + in(f->fuhj, k, L);
      FY[L] = SAAY[L] * FY[L] + in(f->fvhj, k, L);
      L = std::max(1, c->lberc[ll]);
      FX[L] = SAAX[L] * FX[L] + in(f->fuhj, k, L);
      L = std::max(1, c->lbnrc[ll]);
      FY[L] = SAAY[L] * FY[L] + in(f->fvhj, k, L);
    }
  // :797-811 horizontal momentum diffusion
  if (p->ishdmf >= 1)
    for (int k = 0; k < kc; ++k) {
      F<double> FX = K_(c->fx, k), FY = K_(c->fy, k);
      for (int L : lwet) {
        if (!c->lhdmf[L]) continue;
        FX[L] = FX[L] - c->sdx[L] * (in(f->fmdux, k, L) + in(f->fmduy, k, L));
        FY[L] = FY[L] - c->sdy[L] * (in(f->fmdvx, k, L) + in(f->fmdvy, k, L));
      }
    }
  // :940-956 the depth sums
  for (int k = 0; k < kc; ++k) {
    F<double> FCAX = K_(c->fcax, k), FCAY = K_(c->fcay, k), FX = K_(c->fx, k),
              FY = K_(c->fy, k);
    F<double> SGZU{c->msgzu.data() + size_t(k) * n1 + 1},
        SGZV{c->msgzv.data() + size_t(k) * n1 + 1};
    for (int L : lwet) {
      FCAXE[L] = FCAXE[L] + FCAX[L] * SGZU[L];
      FCAYE[L] = FCAYE[L] + FCAY[L] * SGZV[L];
      FXE[L] = FXE[L] + FX[L] * SGZU[L];
      FYE[L] = FYE[L] + FY[L] * SGZV[L];
    }
  }
  for (int k = 0; k < kc; ++k)
    for (int L = 1; L <= lc; ++L) {
      const size_t o = size_t(k) * cld + L - 1;
      if (f->fcax) f->fcax[o] = K_(c->fcax, k)[L];
      if (f->fcay) f->fcay[o] = K_(c->fcay, k)[L];
      if (f->fx) f->fx[o] = K_(c->fx, k)[L];
      if (f->fy) f->fy[o] = K_(c->fy, k)[L];
      if (f->cac) f->cac[o] = K_(c->cac, k)[L];
    }
  return EFDC_XM_OK;
}

int oracle_congrad(oracle_ctx *c, const double *ccc, const double *ccs,
                   const double *ccn, const double *ccw, const double *cce,
                   const double *ccci, const double *fptmp, double *p,
                   double rsqm, int iterm, int *iters, double *rsq) {
  const int lc = c->lc;
  for (int L = 1; L <= lc; ++L) {
    c->ccc[L] = ccc[L - 1];
    c->ccs[L] = ccs[L - 1];
    c->ccn[L] = ccn[L - 1];
    c->ccw[L] = ccw[L - 1];
    c->cce[L] = cce[L - 1];
    c->ccci[L] = ccci[L - 1];
    c->fptmp[L] = fptmp[L - 1];
  }
  int it = 0;
  double r = 0.;
  const int s = congrad(c, F<double>{p}, rsqm, iterm, &it, &r);
  if (iters) *iters = it;
  if (rsq) *rsq = r;
  return s;
}

}  // extern "C"
