// xm_chan.cu -- sub-grid channels (host-guest channel interactions) of
// CALPUV2C: SUBCHAN (subchan.f90:1-124), the couplings CONGRADC adds to the
// CG (congradc.f90:59-116), the new exchange flows (calpuv2c.f90:440-460) and
// the exchange volumes (:538-556).
//
// Channels are few (tens to hundreds per basin): one thread per member walks
// its channels in the reference's NMD order, so every cell's sums round as
// the serial Fortran loops do (compiled without FMA contraction, like the
// other FP64 step kernels).  The CG couplings are applied by small kernels
// between a CG kernel and its member reduction: they correct the cell values
// of the two channel cells and add the change of the cell's dot-product term
// to the partial sum of the quad that holds the cell.
//
// The MIXED form refines towards the system the reference's CONGRADC
// converges to.  CONGRADC adds +CCCCHH both to its initial residual and to
// A*p, so its CG iterates with A+C from a residual of A-C; at convergence
// (A+C)P = b + 2C*P0 with P0 the P at entry.  The FP64 residual of the MIXED
// solve is therefore r = b - A*P + CCCCHH*(2*P0 - P) at the partner cell, and
// its FP32 operator carries +CCCCHH.  With chan_consistent the system is the
// conductance form (A-C)P = b: r = b - A*P + CCCCHH*P and -CCCCHH in A*p.
#include "xm_cg.cuh"
#include "xm_kernels.h"

namespace xm {

#define MEMBER_LOOP                                                                    \
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < S.nmember;                   \
       m += gridDim.x * blockDim.x)

constexpr int CH_NT = 128;  // threads per CTA of the member kernels

// calpuv2c.f90:139-145 (QCHANUT = QCHANU) and :259 (P1 = P) at the channels.
// CALPUV9C (calpuv9c.f90:128-141): QCHANUT = QCHANUN, and for ISTL_ = 3
// QCHANUN = QCHANU; its P1 is P at entry after the advance of ISTL_ = 3, the
// caller's P1 for ISTL_ = 2.
__global__ void k_chan_entry(DevStatic S, DevState X, const int *act) {
  const DevChan &C = S.ch;
  MEMBER_LOOP {
    if (!act[m]) continue;
    const int istl = S.sc[m].istl;
    const double *P1 = istl == 2 ? X.p1 : X.p;
    for (int k = C.cstart[m]; k < C.cstart[m + 1]; ++k) {
      if (istl == 0) {
        C.qut[k] = C.qu[k];
        C.qvt[k] = C.qv[k];
      } else {
        C.qut[k] = C.qun[k];
        C.qvt[k] = C.qvn[k];
        if (istl == 3) {
          C.qun[k] = C.qu[k];
          C.qvn[k] = C.qv[k];
        }
      }
      C.p1h[k] = P1[C.host[k]];
      C.p1g[k] = P1[C.guest[k]];
    }
  }
}

// SUBCHAN (subchan.f90:18-121) for the members in the sweep: activity,
// CCCCHU, CCCCHV, CCCCHH and their entries in CC and FP of the host and guest
// cells (after SETOPENBC, calpuv2c.f90:349-356); then the final CC of the
// channels' cells into the member's minimum diagonal.  In the first sweep HP
// is still the entry value (the view hp0).  first_sweep < 0: the member's
// own sweep counter tells (a step whose sweep loop runs on the device).
__global__ void k_chan_sub(DevStatic S, DevState X, Ctl *ctl, const int *act, int first_sweep) {
  const DevChan &C = S.ch;
  MEMBER_LOOP {
    const int k0 = C.cstart[m], k1 = C.cstart[m + 1];
    if (!act[m] || k0 == k1) continue;
    const StepScalars &c = S.sc[m];
    const double G = c.g, DE_T = c.delt, HDRY = c.hdry, RLAMN = c.rlamn;
    const double RLAMO = 1. - RLAMN;
    const double *H1P = X.h1p;
    const bool first = first_sweep < 0 ? ctl[m].sweep == 0 : first_sweep != 0;
    const double *HP = first ? X.hp0 : X.hp;
    for (int k = k0; k < k1; ++k) {
      const int lh = C.host[k], lg = C.guest[k];
      double cu = 0.0, cv = 0.0;
      int iact = 0;
      const double SRFHOST = H1P[lh] + S.belv[lh];
      const double SRFCHAN = H1P[lg] + S.belv[lg];
      if (C.type[k] == 1) {  // :29-62 x-direction channel
        if (SRFCHAN > SRFHOST)
          if (H1P[lg] > HDRY) iact = 1;
        if (SRFHOST > SRFCHAN)
          if (H1P[lh] > HDRY) iact = 1;
        if (HP[lh] <= 0.0 || HP[lg] <= 0.0)
          if (iact == 1) iact = 0;
        if (iact == 1) {
          const double WCHAN = C.gw[k];
          const double RLCHN = 0.5 * C.gl[k] + C.len[k];
          double HCHAN = 0.5 * C.gl[k] * H1P[lg] + C.len[k] * H1P[lh];
          HCHAN = HCHAN / RLCHN;
          if (HCHAN > 0.) {
            const double TMPVAL = C.fric[k] * DE_T / (HCHAN * HCHAN * WCHAN);
            cu = 1. / (1. + TMPVAL * fabs(C.qut[k]));
            cv = DE_T * HCHAN * WCHAN / RLCHN;
          }
        }
      } else {  // :64-101 y-direction channel
        int IHCHMX = 0, IHCHMN = 0;
        double HCHNMX = 0., HCHNMN = 0.;
        if (SRFCHAN > SRFHOST)
          if (H1P[lg] > HDRY) {
            HCHNMX = -H1P[lg];
            IHCHMX = 1;
            iact = 1;
          }
        if (SRFHOST > SRFCHAN)
          if (H1P[lh] > HDRY) {
            HCHNMN = H1P[lh];
            IHCHMN = 1;
            iact = 1;
          }
        // :84 tests HP(LMDCHU) for the y-direction channel too (L = 1 there
        // unless the input gives a cell)
        const double hpu = C.gu[k] < 0 ? C.hp1[m] : HP[C.gu[k]];
        if (HP[lh] <= 0.0 || hpu <= 0.0)
          if (iact == 1) iact = 0;
        if (iact == 1) {
          const double WCHAN = C.gw[k];
          const double RLCHN = 0.5 * C.gl[k] + C.len[k];
          double HCHAN = 0.5 * C.gl[k] * H1P[lg] + C.len[k] * H1P[lh];
          HCHAN = HCHAN / RLCHN;
          if (IHCHMX == 1) HCHAN = fmax(HCHAN, HCHNMX);
          if (IHCHMN == 1) HCHAN = fmin(HCHAN, HCHNMN);
          if (HCHAN > 0.) {
            const double TMPVAL = C.fric[k] * DE_T / (HCHAN * HCHAN * WCHAN);
            cu = 1. / (1. + TMPVAL * fabs(C.qvt[k]));
            cv = DE_T * HCHAN * WCHAN / RLCHN;
          }
        }
      }
      C.iact[k] = iact;
      C.cu[k] = cu;
      C.cv[k] = cv;
      // :104-119
      X.cc[lh] = X.cc[lh] + G * RLAMN * RLAMN * cu * cv;
      C.chh[k] = G * RLAMN * RLAMN * cu * cv;
      X.cc[lg] = X.cc[lg] + G * RLAMN * RLAMN * cu * cv;
      const double qt = C.type[k] == 1 ? C.qut[k] : C.qvt[k];
      const double TMPVAL = G * (RLAMO + RLAMN * cu) * qt -
                            G * RLAMN * RLAMO * cu * cv * (C.p1h[k] - C.p1g[k]);
      X.fp[lh] = X.fp[lh] + TMPVAL;
      X.fp[lg] = X.fp[lg] - TMPVAL;
    }
    // CC only grows here, so the minimum takes the final values (:360-368)
    for (int k = k0; k < k1; ++k) {
      atomic_min_nonneg(&ctl[m].ccmnm_int, X.cc[C.host[k]]);
      atomic_min_nonneg(&ctl[m].ccmnm_int, X.cc[C.guest[k]]);
    }
  }
}

__device__ __forceinline__ double ccmnmi_of(const Ctl &k) {
  return 1. / fmin(k.ccmnm_int, k.ccmnm_bc);
}

// FP64 CONGRADC, initial residual (congradc.f90:59-77): RCG(guest) +=
// CCCCHH*P(host), RCG(host) += CCCCHH*P(guest) with CCCCHH scaled like the
// system (calpuv2c.f90:401-405); then PCG = RCG*CCCI at those cells and the
// change of RCG*PCG into the quads' partial sums.
__global__ void k_chan_res64(DevStatic S, DevSystem Y, const double *P, const Ctl *ctl,
                             double *part) {
  const DevChan &C = S.ch;
  MEMBER_LOOP {
    const int k0 = C.cstart[m], k1 = C.cstart[m + 1];
    if (k0 == k1 || ctl[m].done) continue;
    const double CCMNMI = ccmnmi_of(ctl[m]);
    auto add = [&](int d, int q, double term) {
      const double r0 = Y.r[d], z0 = Y.pa[d];
      const double r = r0 + term;
      const double z = r * rcpT(Y.ccc[d]);
      Y.r[d] = r;
      Y.pa[d] = z;
      Y.z[d] = z;
      part[q] += r * z - r0 * z0;
    };
    for (int k = k0; k < k1; ++k) {
      const double h = C.chh[k] * CCMNMI;
      add(C.guest[k], C.qguest[k], h * P[C.host[k]]);
      add(C.host[k], C.qhost[k], h * P[C.guest[k]]);
    }
  }
}

// FP64 CONGRADC, A*p (congradc.f90:99-116): APCG(guest) += CCCCHH*PCG(host),
// APCG(host) += CCCCHH*PCG(guest) (-CCCCHH with chan_consistent), and the
// change of APCG*PCG into the quads' partial sums.
__global__ void k_chan_mv64(DevStatic S, DevSystem Y, const Ctl *ctl, double *part) {
  const DevChan &C = S.ch;
  MEMBER_LOOP {
    const int k0 = C.cstart[m], k1 = C.cstart[m + 1];
    if (k0 == k1 || ctl[m].done) continue;
    const double CCMNMI = ccmnmi_of(ctl[m]);
    const bool consistent = S.sc[m].chan_consistent != 0;
    const double *p = ctl[m].parity ? Y.pa : Y.pb;  // the new search direction
    auto add = [&](int d, int q, double term) {
      const double a0 = Y.ap[d];
      const double a = a0 + term;
      Y.ap[d] = a;
      part[q] += (a - a0) * p[d];
    };
    for (int k = k0; k < k1; ++k) {
      const double hs = C.chh[k] * CCMNMI;
      const double h = consistent ? -hs : hs;
      add(C.guest[k], C.qguest[k], h * p[C.host[k]]);
      add(C.host[k], C.qhost[k], h * p[C.guest[k]]);
    }
  }
}

// calpuv2c.f90:440-460: the new exchange flows from the solved P.
__global__ void k_chan_flow(DevStatic S, DevState X, const int *act) {
  const DevChan &C = S.ch;
  MEMBER_LOOP {
    if (!act[m]) continue;
    const double RLAMN = S.sc[m].rlamn, RLAMO = 1. - RLAMN;
    for (int k = C.cstart[m]; k < C.cstart[m + 1]; ++k) {
      if (C.iact[k] > 0) {
        const int lh = C.host[k], lg = C.guest[k];
        const double qt = C.type[k] == 1 ? C.qut[k] : C.qvt[k];
        const double q = C.cu[k] * qt - RLAMN * C.cu[k] * C.cv[k] * (X.p[lh] - X.p[lg]) -
                         RLAMO * C.cu[k] * C.cv[k] * (C.p1h[k] - C.p1g[k]);
        if (C.type[k] == 1) {
          C.qu[k] = q;
          C.qv[k] = 0.;
        } else {
          C.qu[k] = 0.;
          C.qv[k] = q;
        }
      } else {
        C.qv[k] = 0.;
        C.qvn[k] = 0.;
        C.qu[k] = 0.;
        C.qun[k] = 0.;
      }
    }
  }
}

// calpuv2c.f90:538-556: the exchange volumes of the active channels.
__global__ void k_chan_exch(DevStatic S, DevState X, const int *act) {
  const DevChan &C = S.ch;
  MEMBER_LOOP {
    if (!act[m]) continue;
    const StepScalars &c = S.sc[m];
    const double RLAMN = c.rlamn, RLAMO = 1. - RLAMN;
    for (int k = C.cstart[m]; k < C.cstart[m + 1]; ++k) {
      if (C.iact[k] <= 0) continue;
      const int lh = C.host[k], lg = C.guest[k];
      const double q = C.type[k] == 1 ? C.qu[k] : C.qv[k];
      const double qt = C.type[k] == 1 ? C.qut[k] : C.qvt[k];
      const double TMPVAL = c.delt * (RLAMN * q + RLAMO * qt);
      X.hp[lh] = X.hp[lh] + TMPVAL * S.dxyip[lh];
      X.hp[lg] = X.hp[lg] - TMPVAL * S.dxyip[lg];
    }
  }
}

// MIXED: P at the entry of the solve and the FP32 coupling of the
// Jacobi-scaled operator, +-CCCCHH*D(host)*D(guest), for the system V.
__global__ void k_chan_p0(DevStatic S, SysView V, const double *P, const int *act) {
  const DevChan &C = S.ch;
  MEMBER_LOOP {
    if (!act[m]) continue;
    const bool consistent = S.sc[m].chan_consistent != 0;
    for (int k = C.cstart[m]; k < C.cstart[m + 1]; ++k) {
      const int lh = C.host[k], lg = C.guest[k];
      C.p0h[k] = P[lh];
      C.p0g[k] = P[lg];
      const double h = consistent ? -C.chh[k] : C.chh[k];
      C.hh32[k] = float(h * inv_sqrt_diag(V.cc[lh]) * inv_sqrt_diag(V.cc[lg]));
    }
  }
}

// The FP64 residual of the 5-point system V at cell d, as residual_row forms it.
__device__ __forceinline__ double residual_cell(const DevStatic &S, const SysView &V,
                                                const double *P, int d, bool asym) {
  const Nb q = neighbours_of_slot(S.tnbr, d);
  const double kn = asym ? V.cn[d] : V.cs[q.n];
  const double ke = asym ? V.ce[d] : V.cw[q.e];
  return V.fp[d] - V.cc[d] * P[d] - kn * P[q.n] - V.cs[d] * P[q.s] - V.cw[d] * P[q.w] -
         ke * P[q.e];
}

// MIXED: the channel terms of the FP64 refinement residual at the channels'
// cells (r += CCCCHH*(2*P0 - P) of the partner, or CCCCHH*P with
// chan_consistent), the scaled FP32 residual there, and the changes of both
// sums (r.r, r32.r32) into the quads' partial sums.
__global__ void k_chan_resmx(DevStatic S, SysView V, DevSystem Y, const double *P,
                             const Ctl *ctl, double *part) {
  const DevChan &C = S.ch;
  MEMBER_LOOP {
    const int k0 = C.cstart[m], k1 = C.cstart[m + 1];
    if (k0 == k1 || ctl[m].done) continue;
    const bool asym = (ctl[m].asym & 1) != 0;
    const bool consistent = S.sc[m].chan_consistent != 0;
    auto term = [&](int j, bool at_host) {  // channel j's term at its host or guest cell
      const double pp = at_host ? P[C.guest[j]] : P[C.host[j]];
      const double p0 = at_host ? C.p0g[j] : C.p0h[j];
      return consistent ? C.chh[j] * pp : C.chh[j] * (2.0 * p0 - pp);
    };
    auto fix = [&](int d, int q) {  // every channel term at cell d, in NMD order
      const double r5 = residual_cell(S, V, P, d, asym);
      double r = r5;
      for (int j = k0; j < k1; ++j) {
        if (C.guest[j] == d) r += term(j, false);
        if (C.host[j] == d) r += term(j, true);
      }
      const float r32o = Y.r32[d];
      const float r32n = float(r * inv_sqrt_diag(V.cc[d]));
      Y.r32[d] = r32n;
      Y.pa32[d] = r32n;
      part[q] += r * r - r5 * r5;
      part[size_t(S.nquad) + q] +=
          double(r32n) * double(r32n) - double(r32o) * double(r32o);
    };
    for (int k = k0; k < k1; ++k) {  // each channel cell once
      if (C.first_guest[k]) fix(C.guest[k], C.qguest[k]);
      if (C.first_host[k]) fix(C.host[k], C.qhost[k]);
    }
  }
}

// MIXED: the FP32 couplings in Ahat*p and the change of p.Ap into the quads'
// partial sums.
__global__ void k_chan_mvmx(DevStatic S, DevSystem Y, const Ctl *ctl, double *part) {
  const DevChan &C = S.ch;
  MEMBER_LOOP {
    const int k0 = C.cstart[m], k1 = C.cstart[m + 1];
    if (k0 == k1 || (ctl[m].done | ctl[m].idone)) continue;
    const float *p = ctl[m].parity ? Y.pa32 : Y.pb32;  // the new search direction
    auto add = [&](int d, int q, float term) {
      const float a0 = Y.ap32[d];
      const float a = a0 + term;
      Y.ap32[d] = a;
      part[q] += (double(a) - double(a0)) * double(p[d]);
    };
    for (int k = k0; k < k1; ++k) {
      const float h = C.hh32[k];
      add(C.guest[k], C.qguest[k], h * p[C.host[k]]);
      add(C.host[k], C.qhost[k], h * p[C.guest[k]]);
    }
  }
}

static int member_grid(const DevStatic &S) { return (S.nmember + CH_NT - 1) / CH_NT; }

void launch_chan_entry(const Launch &l, const DevStatic &S, const DevState &X, const int *act) {
  if (!l.chan) return;
  k_chan_entry<<<member_grid(S), CH_NT, 0, l.stream>>>(S, X, act);
  count_launches(1);
}
void launch_chan_sub(const Launch &l, const DevStatic &S, const DevState &X, Ctl *ctl,
                     const int *act, int first_sweep) {
  if (!l.chan) return;
  k_chan_sub<<<member_grid(S), CH_NT, 0, l.stream>>>(S, X, ctl, act, first_sweep);
  count_launches(1);
}
void launch_chan_res64(const Launch &l, const DevStatic &S, const DevSystem &Y, const double *P,
                       const Ctl *ctl, double *part) {
  if (!l.chan) return;
  k_chan_res64<<<member_grid(S), CH_NT, 0, l.stream>>>(S, Y, P, ctl, part);
  count_launches(1);
}
void launch_chan_mv64(const Launch &l, const DevStatic &S, const DevSystem &Y, const Ctl *ctl,
                      double *part) {
  if (!l.chan) return;
  k_chan_mv64<<<member_grid(S), CH_NT, 0, l.stream>>>(S, Y, ctl, part);
  count_launches(1);
}
void launch_chan_flow(const Launch &l, const DevStatic &S, const DevState &X, const int *act) {
  if (!l.chan) return;
  k_chan_flow<<<member_grid(S), CH_NT, 0, l.stream>>>(S, X, act);
  count_launches(1);
}
void launch_chan_exch(const Launch &l, const DevStatic &S, const DevState &X, const int *act) {
  if (!l.chan) return;
  k_chan_exch<<<member_grid(S), CH_NT, 0, l.stream>>>(S, X, act);
  count_launches(1);
}
void launch_chan_p0(const Launch &l, const DevStatic &S, const SysView &V, const double *P,
                    const int *act) {
  if (!l.chan) return;
  k_chan_p0<<<member_grid(S), CH_NT, 0, l.stream>>>(S, V, P, act);
  count_launches(1);
}
void launch_chan_resmx(const Launch &l, const DevStatic &S, const SysView &V, const DevSystem &Y,
                       const double *P, const Ctl *ctl, double *part) {
  if (!l.chan) return;
  k_chan_resmx<<<member_grid(S), CH_NT, 0, l.stream>>>(S, V, Y, P, ctl, part);
  count_launches(1);
}
void launch_chan_mvmx(const Launch &l, const DevStatic &S, const DevSystem &Y, const Ctl *ctl,
                      double *part) {
  if (!l.chan) return;
  k_chan_mvmx<<<member_grid(S), CH_NT, 0, l.stream>>>(S, Y, ctl, part);
  count_launches(1);
}

}  // namespace xm
