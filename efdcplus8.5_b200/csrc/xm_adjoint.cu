// xm_adjoint.cu -- calibration support: the bottom drag of the calibration
// model, and the reverse (adjoint) of one external-mode step.
//
// The calibration model is the CALPUV2C step (calpuv2c.f90:128-1187) with
// ISDRY=0 and clamped open boundaries (ISPB=0), preceded by the bottom
// stress the step reads as TBX/TBY, written here from a per-cell Manning n:
//   TBX = STBX*SQRT(VU^2 + U^2)*U,  STBX = G*n_u^2/HU^(1/3)
// (the form of hdmt2t.f90:682 with AVCON1=0 and a Manning drag coefficient;
// U = UHDYE*DYIU/HU is the depth-averaged u-face velocity, VU the mean of
// the four v-face velocities around the u face, n_u the mean n of the two
// cells of the face; TBY alike).
//
// Reverse of one step, given the adjoints of its outputs (P, HP, HU, HV,
// UHDYE, VHDXE after the step) and the step's start state and CG solution P':
//   k_adj_hpe    HU/HV = (DXYP*HP + DXYP_W*HP_W)*0.5/DXYU and P = G*(HP+BELV)
//                (calpuv2c.f90:896-906) -> adjoint of HP'
//   k_adj_pre    continuity (:466-486), the boundary depths (:489-535) and the
//                back-substitution (:416-437) -> rhs of the adjoint solve
//   (CONGRAD)    A*lambda = rhs on the step's own operator: A is symmetric
//                with clamped boundaries, so the adjoint solve is the same CG
//   k_adj_coef   coefficients (:306-344, SETOPENBC2) -> HU/HV; FP -> lambda
//   k_adj_obc    SETOPENBC targets (setopenbc.f90:22-206) -> PCB/PSB
//   k_adj_fp     FP, FP1, FUHDYE/FVHDXE (:214-220, :282-290, :306-314) and
//                the drag -> P, UHDYE/VHDXE, HU/HV, Manning n
//   k_adj_gath   the neighbour sums of the drag (n_u, VU, UV)
// Each face coefficient w (CW(L) = CE(LW) = w, CC(L) and CC(LW) minus w)
// gets d(loss)/dw = (l_L - l_W)*(P'_L - P'_W), with l = lambda on interior
// rows and 0 on boundary rows (their rows are fixed by SETOPENBC).

#include "xm_common.cuh"
#include "xm_kernels.h"

namespace xm {

#define TILE_LOOP(ntile) for (int tile = blockIdx.x + 1; tile < (ntile); tile += gridDim.x)

namespace {

// depth-averaged face velocities of a state (0 at land slots)
__device__ __forceinline__ double vel_u(const DevStatic &S, const double *uh, const double *hu,
                                        int x) {
  return S.kind[x] == LAND ? 0.0 : uh[x] * S.dyiu[x] / hu[x];
}
__device__ __forceinline__ double vel_v(const DevStatic &S, const double *vh, const double *hv,
                                        int x) {
  return S.kind[x] == LAND ? 0.0 : vh[x] * S.dxiv[x] / hv[x];
}

}  // namespace

// Drag of the calibration model from the state in A.u0/v0/hu0/hv0.
__global__ void __launch_bounds__(NT) k_cal_tbxy(DevStatic S, DevCalib A, int ntile) {
  TILE_LOOP(ntile) {
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    const double g = S.sc[0].g;
    double tbx = 0.0, tby = 0.0;
    if (S.subo[d] > 0.5) {
      const int nw = neighbours_of_slot(S.tnbr, q.w).n;
      const double U = vel_u(S, A.u0, A.hu0, d);
      const double VU = 0.25 * (vel_v(S, A.v0, A.hv0, d) + vel_v(S, A.v0, A.hv0, q.n) +
                                vel_v(S, A.v0, A.hv0, q.w) + vel_v(S, A.v0, A.hv0, nw));
      const double nu = 0.5 * (exp(A.kappa[d]) + exp(A.kappa[q.w]));
      const double stbx = g * nu * nu / cbrt(A.hu0[d]);
      tbx = stbx * sqrt(VU * VU + U * U) * U;
    }
    if (S.svbo[d] > 0.5) {
      const int se = neighbours_of_slot(S.tnbr, q.s).e;
      const double V = vel_v(S, A.v0, A.hv0, d);
      const double UV = 0.25 * (vel_u(S, A.u0, A.hu0, d) + vel_u(S, A.u0, A.hu0, q.e) +
                                vel_u(S, A.u0, A.hu0, q.s) + vel_u(S, A.u0, A.hu0, se));
      const double nv = 0.5 * (exp(A.kappa[d]) + exp(A.kappa[q.s]));
      const double stby = g * nv * nv / cbrt(A.hv0[d]);
      tby = stby * sqrt(UV * UV + V * V) * V;
    }
    A.tbx[d] = tbx;
    A.tby[d] = tby;
  }
}

// Adjoint of HP' from P = G*(HP'+BELV) and the face depths; BELV gradient.
__global__ void __launch_bounds__(NT) k_adj_hpe(DevStatic S, DevCalib A, int ntile) {
  TILE_LOOP(ntile) {
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    const double g = S.sc[0].g;
    const double ap = A.ap_in[d];
    A.ahpe[d] = A.ahp_in[d] + g * ap +
                S.dxyp[d] * (S.fsgzu[d] * A.ahu_in[d] + S.fsgzu[q.e] * A.ahu_in[q.e] +
                             S.fsgzv[d] * A.ahv_in[d] + S.fsgzv[q.n] * A.ahv_in[q.n]);
    A.abelv[d] += g * ap;
  }
}

// Continuity, boundary depths and back-substitution: the outputs' adjoints
// of the old fluxes and H1P, the first HU/HV terms, FUHDYE/FVHDXE's adjoint
// through UHDYE/VHDXE, and the rhs of the adjoint solve (d(loss)/dP').
__global__ void __launch_bounds__(NT) k_adj_pre(DevStatic S, DevState X, DevCalib A, int ntile) {
  TILE_LOOP(ntile) {
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    const uint8_t kd = S.kind[d];
    if (kd == LAND) continue;
    const StepScalars &c = S.sc[0];
    const double D2 = c.deltd2;
    auto hpe = [&](int x) { return S.kind[x] == WATER ? A.ahpe[x] : 0.0; };
    const double hd = hpe(d);
    // the continuity equation's face terms (the same for UHDYE' and UHDY1E)
    const double cu = D2 * (S.dxyip[d] * hd - S.dxyip[q.w] * hpe(q.w));
    const double cv = D2 * (S.dxyip[d] * hd - S.dxyip[q.s] * hpe(q.s));
    const double cue = D2 * (S.dxyip[q.e] * hpe(q.e) - S.dxyip[d] * hd);
    const double cvn = D2 * (S.dxyip[q.n] * hpe(q.n) - S.dxyip[d] * hd);
    const double aun = A.au_in[d] + cu, avn = A.av_in[d] + cv;
    const double aune = A.au_in[q.e] + cue, avnn = A.av_in[q.n] + cvn;
    auto au_ = [&](int x) { return X.sub[x] * D2 * S.hruo[x] * X.rcx[x] * A.hu0[x]; };
    auto av_ = [&](int x) { return X.svb[x] * D2 * S.hrvo[x] * X.rcy[x] * A.hv0[x]; };
    A.au_out[d] = cu;
    A.av_out[d] = cv;
    A.ahp_out[d] = (kd == WATER) ? A.ahpe[d] : 0.0;
    A.afu[d] = X.sub[d] * aun;
    A.afv[d] = X.svb[d] * avn;
    A.ahu_out[d] = -X.sub[d] * D2 * S.hruo[d] * X.rcx[d] * (A.psol[d] - A.psol[q.w]) * aun;
    A.ahv_out[d] = -X.svb[d] * D2 * S.hrvo[d] * X.rcy[d] * (A.psol[d] - A.psol[q.s]) * avn;
    double rhs = -au_(d) * aun + au_(q.e) * aune - av_(d) * avn + av_(q.n) * avnn;
    if (kd == OPENBC) {  // HP' = P'/G - BELV on the boundary cells
      rhs += A.ahpe[d] * c.gi;
      A.abelv[d] -= A.ahpe[d];
    }
    A.rhs[d] = rhs;
  }
}

// rhs of the adjoint solve in the scaled system (FPTMP = rhs/CCMNM), zero
// initial guess, and sum(rhs_scaled^2) into *bsq for the relative stop.
__global__ void __launch_bounds__(NT) k_adj_rhs(DevStatic S, DevSystem Y, const Ctl *ctl,
                                               DevCalib A, int ntile, double *bsq) {
  __shared__ double sh[32];
  const double ccmnmi = 1. / fmin(ctl[0].ccmnm_int, ctl[0].ccmnm_bc);
  double acc = 0.0;
  TILE_LOOP(ntile) {
    const int d = tile * TILE + threadIdx.x;
    const double b = (S.kind[d] == LAND) ? 0.0 : A.rhs[d] * ccmnmi;
    Y.fptmp[d] = b;
    A.lam[d] = 0.0;
    acc += b * b;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) atomicAdd(bsq, acc);
}

// Coefficient adjoints from lambda and P' -> HU/HV; adjoint of FP.
__global__ void __launch_bounds__(NT) k_adj_coef(DevStatic S, DevState X, DevCalib A, int ntile) {
  TILE_LOOP(ntile) {
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    const StepScalars &c = S.sc[0];
    const double C1 = -0.5 * c.deltd2 * c.g;
    auto lt = [&](int x) { return S.kind[x] == WATER ? A.lam[x] : 0.0; };
    const double ld = lt(d);
    const double wu = (ld - lt(q.w)) * (A.psol[d] - A.psol[q.w]);
    const double wv = (ld - lt(q.s)) * (A.psol[d] - A.psol[q.s]);
    A.ahu_out[d] += C1 * X.sub[d] * S.hruo[d] * X.rcx[d] * wu;
    A.ahv_out[d] += C1 * X.svb[d] * S.hrvo[d] * X.rcy[d] * wv;
    A.afp[d] = ld;
  }
}

// Boundary targets: d(loss)/d(fp) = lambda_bc*DELTI*DXYP + lambda_nb*CT,
// accumulated onto the harmonic amplitudes PCB/PSB.
__global__ void k_adj_obc(DevStatic S, DevState X, DevObc B, DevCalib A) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < B.n; k += gridDim.x * blockDim.x) {
    const StepScalars &c = S.sc[0];
    const int d = B.slot[k], nb = B.nbr[k], side = B.side[k];
    const int mt = B.mtide[0];
    double fp = B.pser ? B.pser[k] : 0.0;
    for (int t = 0; t < mt; ++t)
      fp = fp + B.pcb[k * B.mtmax + t] * c.cosv[t] + B.psb[k * B.mtmax + t] * c.sinv[t];
    const double FP1G = fp / c.g - 0.2 * c.hdry;
    if (FP1G < S.belv[d] || FP1G < S.belv[nb]) {  // dry-clamped target: a constant
      atomicAdd(A.nflag, 1);
      continue;
    }
    const double D = c.deltd2, G = c.g;
    double CT;
    if (side == 0)
      CT = 0.5 * D * G * S.hruo[nb] * X.rcx[nb] * A.hu0[nb];
    else if (side == 1)
      CT = 0.5 * D * G * S.hruo[d] * X.rcx[d] * A.hu0[d];
    else if (side == 2)
      CT = 0.5 * D * G * S.hrvo[nb] * X.rcy[nb] * A.hv0[nb];
    else
      CT = 0.5 * D * G * S.hrvo[d] * X.rcy[d] * A.hv0[d];
    const double fbar = A.lam[d] * c.delti * S.dxyp[d] + A.lam[nb] * CT;
    for (int t = 0; t < mt; ++t) {
      A.apcb[k * B.mtmax + t] += fbar * c.cosv[t];
      A.apsb[k * B.mtmax + t] += fbar * c.sinv[t];
    }
  }
}

// FP -> FP1, FUHDYE/FVHDXE; FP1 and FUHDYE/FVHDXE -> P, UHDYE/VHDXE, HU/HV,
// TBX/TBY; TBX/TBY -> the face velocities, HU/HV and the face Manning n.
__global__ void __launch_bounds__(NT) k_adj_fp(DevStatic S, DevState X, DevCalib A, int ntile) {
  TILE_LOOP(ntile) {
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    const StepScalars &c = S.sc[0];
    const double D2 = c.deltd2, g = c.g;
    auto afu_t = [&](int x, int xw) {
      return A.afu[x] + 0.5 * g * X.sub[x] * (A.afp[x] - A.afp[xw]);
    };
    auto afv_t = [&](int x, int xs) {
      return A.afv[x] + 0.5 * g * X.svb[x] * (A.afp[x] - A.afp[xs]);
    };
    const double fu = afu_t(d, q.w), fv = afv_t(d, q.s);
    const double fue = afu_t(q.e, d), fvn = afv_t(q.n, d);
    A.ap_out[d] = c.delti * S.dxyp[d] * A.afp[d] - D2 * X.sub[d] * S.hruo[d] * A.hu0[d] * fu +
                  D2 * X.sub[q.e] * S.hruo[q.e] * A.hu0[q.e] * fue -
                  D2 * X.svb[d] * S.hrvo[d] * A.hv0[d] * fv +
                  D2 * X.svb[q.n] * S.hrvo[q.n] * A.hv0[q.n] * fvn;
    double au = fu + 0.5 * g * (A.afp[d] - A.afp[q.w]);
    double av = fv + 0.5 * g * (A.afp[d] - A.afp[q.s]);
    double ahu = -D2 * X.sub[d] * S.hruo[d] * (A.p0[d] - A.p0[q.w]) * fu;
    double ahv = -D2 * X.svb[d] * S.hrvo[d] * (A.p0[d] - A.p0[q.s]) * fv;
    const double tbxb = -X.sub[d] * c.delt * S.dxiu[d] * S.dxyu[d] * c.ritb1 * fu;
    const double tbyb = -X.svb[d] * c.delt * S.dyiv[d] * S.dxyv[d] * c.ritb1 * fv;
    double nbu = 0.0, vub = 0.0, nbv = 0.0, uvb = 0.0;
    if (S.subo[d] > 0.5) {  // TBX = STBX*s*U
      const int nw = neighbours_of_slot(S.tnbr, q.w).n;
      const double hu = A.hu0[d];
      const double U = vel_u(S, A.u0, A.hu0, d);
      const double VU = 0.25 * (vel_v(S, A.v0, A.hv0, d) + vel_v(S, A.v0, A.hv0, q.n) +
                                vel_v(S, A.v0, A.hv0, q.w) + vel_v(S, A.v0, A.hv0, nw));
      const double s = sqrt(VU * VU + U * U);
      const double nu = 0.5 * (exp(A.kappa[d]) + exp(A.kappa[q.w]));
      const double ch = cbrt(hu);
      const double stbx = g * nu * nu / ch;
      const double ub = (s > 0.0) ? tbxb * stbx * (s + U * U / s) : 0.0;
      vub = (s > 0.0) ? tbxb * stbx * U * VU / s : 0.0;
      const double sb = tbxb * s * U;
      nbu = sb * 2.0 * g * nu / ch;
      ahu += -sb * g * nu * nu / (3.0 * ch * hu);
      au += ub * S.dyiu[d] / hu;
      ahu += -ub * A.u0[d] * S.dyiu[d] / (hu * hu);
    }
    if (S.svbo[d] > 0.5) {  // TBY = STBY*s*V
      const int se = neighbours_of_slot(S.tnbr, q.s).e;
      const double hv = A.hv0[d];
      const double V = vel_v(S, A.v0, A.hv0, d);
      const double UV = 0.25 * (vel_u(S, A.u0, A.hu0, d) + vel_u(S, A.u0, A.hu0, q.e) +
                                vel_u(S, A.u0, A.hu0, q.s) + vel_u(S, A.u0, A.hu0, se));
      const double s = sqrt(UV * UV + V * V);
      const double nv = 0.5 * (exp(A.kappa[d]) + exp(A.kappa[q.s]));
      const double ch = cbrt(hv);
      const double stby = g * nv * nv / ch;
      const double vb = (s > 0.0) ? tbyb * stby * (s + V * V / s) : 0.0;
      uvb = (s > 0.0) ? tbyb * stby * V * UV / s : 0.0;
      const double sb = tbyb * s * V;
      nbv = sb * 2.0 * g * nv / ch;
      ahv += -sb * g * nv * nv / (3.0 * ch * hv);
      av += vb * S.dxiv[d] / hv;
      ahv += -vb * A.v0[d] * S.dxiv[d] / (hv * hv);
    }
    A.au_out[d] += au;
    A.av_out[d] += av;
    A.ahu_out[d] += ahu;
    A.ahv_out[d] += ahv;
    A.nbu[d] = nbu;
    A.nbv[d] = nbv;
    A.vub[d] = vub;
    A.uvb[d] = uvb;
  }
}

// The drag's neighbour sums: n_u = (n_L + n_W)/2 -> log n; VU and UV (means
// of four face velocities) -> the velocities of those faces.
__global__ void __launch_bounds__(NT) k_adj_gath(DevStatic S, DevCalib A, int ntile) {
  TILE_LOOP(ntile) {
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    A.akappa[d] += 0.5 * exp(A.kappa[d]) * (A.nbu[d] + A.nbu[q.e] + A.nbv[d] + A.nbv[q.n]);
    // V(d) is in VU(d), VU(LS), VU(LE), VU(LE(LS)); U(d) in UV(d), UV(LW), UV(LN), UV(LN(LW))
    double vb = A.vub[d] + A.vub[q.s] + A.vub[q.e];
    if (S.kind[q.s] != LAND) vb += A.vub[neighbours_of_slot(S.tnbr, q.s).e];
    double ub = A.uvb[d] + A.uvb[q.w] + A.uvb[q.n];
    if (S.kind[q.w] != LAND) ub += A.uvb[neighbours_of_slot(S.tnbr, q.w).n];
    vb *= 0.25;
    ub *= 0.25;
    const double hu = A.hu0[d], hv = A.hv0[d];
    A.au_out[d] += ub * S.dyiu[d] / hu;
    A.ahu_out[d] += -ub * A.u0[d] * S.dyiu[d] / (hu * hu);
    A.av_out[d] += vb * S.dxiv[d] / hv;
    A.ahv_out[d] += -vb * A.v0[d] * S.dxiv[d] / (hv * hv);
  }
}

__global__ void k_adj_gauge(const int *slots, const double *w, int n, double *ap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ap[slots[i]] += w[i];
}

__global__ void k_gather_slots(const double *src, const int *slots, int n, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = src[slots[i]];
}

void launch_cal_tbxy(const Launch &l, const DevStatic &S, const DevState &, const DevCalib &A) {
  k_cal_tbxy<<<l.grid, NT, 0, l.stream>>>(S, A, l.ntile);
  count_launches(1);
}
void launch_adj_gauge(const Launch &l, const int *slots, const double *w, int n, double *ap) {
  if (n <= 0) return;
  k_adj_gauge<<<(n + 255) / 256, 256, 0, l.stream>>>(slots, w, n, ap);
  count_launches(1);
}
void launch_adj_pre(const Launch &l, const DevStatic &S, const DevState &X, const DevObc &,
                    const DevCalib &A) {
  k_adj_hpe<<<l.grid, NT, 0, l.stream>>>(S, A, l.ntile);
  k_adj_pre<<<l.grid, NT, 0, l.stream>>>(S, X, A, l.ntile);
  count_launches(2);
}
void launch_adj_rhs(const Launch &l, const DevStatic &S, const DevSystem &Y, const Ctl *ctl,
                    const DevCalib &A, double *bsq) {
  k_adj_rhs<<<l.grid, NT, 0, l.stream>>>(S, Y, ctl, A, l.ntile, bsq);
  count_launches(1);
}
void launch_adj_post(const Launch &l, const DevStatic &S, const DevState &X, const DevObc &B,
                     const DevCalib &A) {
  k_adj_coef<<<l.grid, NT, 0, l.stream>>>(S, X, A, l.ntile);
  if (B.n > 0) k_adj_obc<<<(B.n + 255) / 256, 256, 0, l.stream>>>(S, X, B, A);
  k_adj_fp<<<l.grid, NT, 0, l.stream>>>(S, X, A, l.ntile);
  k_adj_gath<<<l.grid, NT, 0, l.stream>>>(S, A, l.ntile);
  count_launches(B.n > 0 ? 4 : 3);
}
void launch_gather_slots(cudaStream_t st, const double *src, const int *slots, int n, double *out) {
  if (n <= 0) return;
  k_gather_slots<<<(n + 255) / 256, 256, 0, st>>>(src, slots, n, out);
  count_launches(1);
}

}  // namespace xm
