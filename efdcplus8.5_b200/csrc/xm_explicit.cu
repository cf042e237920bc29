// xm_explicit.cu -- the explicit momentum producer: CALEXP2T's external-mode
// terms (calexp2t.f90:129-956, IS2LMC = 0) on the device.  Compiled with
// -fmad=false and written in the reference's operand order, so every cell's
// FCAXE, FCAYE, FXE, FYE rounds as EFDC+'s FP64 build rounds it.
//
// Layer arrays are [k][slot] (k = K-1, stride MomDev::ls).  Four passes over
// the members' tiles, one CTA per tile and layer (blockIdx.y = k):
//   k_mom_flux   upwind momentum fluxes FUHU, FVHU, FVHV, FUHV (:202-237,
//                STCUV :460-472) and the Coriolis-curvature coefficient CAC
//                with its per-member sum (:481-535);
//   k_mom_accel  FCAX, FCAY (:545-562) and the layer forcings FX, FY
//                (:648-662), which read the neighbours' fluxes and CAC;
//   k_mom_edges  one CTA per member, a thread per layer: the type-2 open
//                boundaries (:605-645) and the flow-boundary edges (:664-689),
//                in the reference's serial order;
//   k_mom_sum    the horizontal momentum diffusion (:797-811) and the depth
//                sums in K order (:940-956) into the step's FCAXE, FCAYE, FXE,
//                FYE.
// Cells outside the wet set (and land slots, which stand for the ghost cell
// LC) hold 0 in every flux, CAC and output array, as the reference's arrays
// of dry cells do after it zeroes them on drying (:131-175).

#include "xm_common.cuh"
#include "xm_kernels.h"

namespace xm {

namespace {

// Fortran MAX(x, 0.) and MIN(x, 0.) in the form std::max / std::min take
__device__ __forceinline__ double max0(double x) { return (x < 0.) ? 0. : x; }
__device__ __forceinline__ double min0(double x) { return (0. < x) ? 0. : x; }

__device__ __forceinline__ bool wet_at(const DevStatic &S, const MomDev &M, int d) {
  return S.kind[d] != LAND && (!M.wet || M.wet[d] != 0);
}

}  // namespace

__global__ void __launch_bounds__(NT) k_mom_flux(DevStatic S, MomDev M, int ntile) {
  __shared__ double sh[32];
  const int k = blockIdx.y;
  const size_t o = size_t(k) * M.ls;
  for (int tile = blockIdx.x + 1; tile < ntile; tile += gridDim.x) {
    const int m = S.tile_member[tile];
    const MomScalars &c = M.sc[m];
    if (!c.on || k >= c.kc) continue;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    double fuhu = 0., fvhu = 0., fvhv = 0., fuhv = 0., cac = 0.;
    if (wet_at(S, M, d)) {
      const double *U = M.u + o, *V = M.v + o, *UH = M.uhdy + o, *VH = M.vhdx + o;
      // :211-232
      const double UHB = 0.5 * (UH[d] + UH[q.e]);
      const double VHC = 0.5 * (VH[d] + VH[q.w]);
      fuhu = max0(UHB) * U[d] + min0(UHB) * U[q.e];
      fvhu = max0(VHC) * U[q.s] + min0(VHC) * U[d];
      const double VHB = 0.5 * (VH[d] + VH[q.n]);
      const double UHC = 0.5 * (UH[d] + UH[q.s]);
      fvhv = max0(VHB) * V[d] + min0(VHB) * V[q.n];
      fuhv = max0(UHC) * V[q.w] + min0(UHC) * V[d];
      if (c.tri) {  // :466-467
        fuhu = M.stcuv[d] * fuhu;
        fvhv = M.stcuv[d] * fvhv;
      }
      if (c.curv)  // :489
        cac = (M.fcorc[d] * S.dxyp[d] + 0.5 * c.snlt * (V[q.n] + V[d]) * M.dydi[d] -
               0.5 * c.snlt * (U[q.e] + U[d]) * M.dxdj[d]) *
              M.hp[d];
    }
    M.fuhu[o + d] = fuhu;
    M.fvhu[o + d] = fvhu;
    M.fvhv[o + d] = fvhv;
    M.fuhv[o + d] = fuhv;
    M.cac[o + d] = cac;
    if (c.curv) {  // CACSUM decides only whether |sum| exceeds 1e-7 (:522, :545)
      const double t = block_sum(cac, sh);
      if (threadIdx.x == 0 && t != 0.) atomicAdd(&M.cacsum[m], t);
    }
  }
}

__global__ void __launch_bounds__(NT) k_mom_accel(DevStatic S, MomDev M, int ntile) {
  const int k = blockIdx.y;
  const size_t o = size_t(k) * M.ls;
  for (int tile = blockIdx.x + 1; tile < ntile; tile += gridDim.x) {
    const int m = S.tile_member[tile];
    const MomScalars &c = M.sc[m];
    if (!c.on || k >= c.kc) continue;
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    double fcax = 0., fcay = 0., fx = 0., fy = 0.;
    if (wet_at(S, M, d)) {
      const double *U = M.u + o, *V = M.v + o, *CAC = M.cac + o;
      if (c.curv && fabs(M.cacsum[m]) > 1.E-7) {  // :545-562
        const int nw = M.nw[d], se = M.se[d];
        fcax = 0.25 * M.scax[d] * (CAC[d] * (V[q.n] + V[d]) + CAC[q.w] * (V[nw] + V[q.w]));
        fcay = 0.25 * M.scay[d] * (CAC[d] * (U[q.e] + U[d]) + CAC[q.s] * (U[se] + U[q.s]));
      }
      // :653-654
      const double *FUHU = M.fuhu + o, *FVHU = M.fvhu + o, *FVHV = M.fvhv + o,
                   *FUHV = M.fuhv + o;
      fx = M.fsgzu[o + d] * (FUHU[d] - FUHU[q.w] + FVHU[q.n] - FVHU[d]) +
           (c.fuhj ? M.fuhj[o + d] : 0.);
      fy = M.fsgzv[o + d] * (FVHV[d] - FVHV[q.s] + FUHV[q.e] - FUHV[d]) +
           (c.fuhj ? M.fvhj[o + d] : 0.);
    }
    if (S.kind[d] != LAND) {
      M.fcax[o + d] = fcax;
      M.fcay[o + d] = fcay;
      M.fx[o + d] = fx;
      M.fy[o + d] = fy;
    }
  }
}

// Entries of the serial lists: type-2 boundaries t2 = (side, slot of L, the
// two neighbour slots the form reads), flow-boundary edges bc = (LBCS,
// LBERC, LBNRC slots; -1 for none).
__global__ void k_mom_edges(DevStatic S, MomDev M) {
  const int m = blockIdx.x;
  const MomScalars &c = M.sc[m];
  if (!c.on) return;
  for (int k = threadIdx.x; k < c.kc; k += blockDim.x) {
    const size_t o = size_t(k) * M.ls;
    const double *U = M.u + o, *V = M.v + o, *CAC = M.cac + o;
    double *FCAX = M.fcax + o, *FCAY = M.fcay + o, *FX = M.fx + o, *FY = M.fy + o;
    for (int j = M.t2start[m]; j < M.t2start[m + 1]; ++j) {
      const int4 e = M.t2[j];
      const int L = e.y, a = e.z, b = e.w;
      switch (e.x) {
        case 0:  // W (:607-614): a = LN
          FCAX[L] = 0.5 * M.scax[L] * CAC[L] * (V[a] + V[L]);
          break;
        case 1:  // E (:617-624): a = LWC, b = LNWC
          FCAX[L] = 0.5 * M.scax[L] * CAC[a] * (V[b] + V[a]);
          break;
        case 2:  // S (:627-633): a = LEC
          FCAY[L] = 0.5 * M.scay[L] * CAC[L] * (U[a] + U[L]);
          break;
        default:  // N (:636-643): a = LSC, b = LSEC
          FCAY[L] = 0.5 * M.scay[L] * CAC[a] * (U[b] + U[a]);
          break;
      }
    }
    for (int j = M.bcstart[m]; j < M.bcstart[m + 1]; ++j) {  // :664-689
      const int4 e = M.bc[j];
      if (e.x >= 0) {
        FX[e.x] = M.saax[e.x] * FX[e.x] + (c.fuhj ? M.fuhj[o + e.x] : 0.);
        FY[e.x] = M.saay[e.x] * FY[e.x] + (c.fuhj ? M.fvhj[o + e.x] : 0.);
      }
      if (e.y >= 0) FX[e.y] = M.saax[e.y] * FX[e.y] + (c.fuhj ? M.fuhj[o + e.y] : 0.);
      if (e.z >= 0) FY[e.z] = M.saay[e.z] * FY[e.z] + (c.fuhj ? M.fvhj[o + e.z] : 0.);
    }
  }
}

__global__ void __launch_bounds__(NT) k_mom_sum(DevStatic S, MomDev M, DevState X, int ntile) {
  for (int tile = blockIdx.x + 1; tile < ntile; tile += gridDim.x) {
    const int m = S.tile_member[tile];
    const MomScalars &c = M.sc[m];
    if (!c.on) continue;
    const int d = tile * TILE + threadIdx.x;
    if (S.kind[d] == LAND) continue;
    double fcaxe = 0., fcaye = 0., fxe = 0., fye = 0.;
    if (!M.wet || M.wet[d]) {
      const bool hd = c.hdmf && M.lhdmf[d];
      for (int k = 0; k < c.kc; ++k) {
        const size_t i = size_t(k) * M.ls + d;
        double fx = M.fx[i], fy = M.fy[i];
        if (hd) {  // :805-806
          fx = fx - M.sdx[d] * (M.fmdux[i] + M.fmduy[i]);
          fy = fy - M.sdy[d] * (M.fmdvx[i] + M.fmdvy[i]);
          M.fx[i] = fx;
          M.fy[i] = fy;
        }
        // :949-952
        fcaxe = fcaxe + M.fcax[i] * M.sgzu[i];
        fcaye = fcaye + M.fcay[i] * M.sgzv[i];
        fxe = fxe + fx * M.sgzu[i];
        fye = fye + fy * M.sgzv[i];
      }
    }
    const_cast<double *>(X.fcaxe)[d] = fcaxe;
    const_cast<double *>(X.fcaye)[d] = fcaye;
    const_cast<double *>(X.fxe)[d] = fxe;
    const_cast<double *>(X.fye)[d] = fye;
  }
}

void launch_explicit(const Launch &l, const DevStatic &S, const MomDev &M, const DevState &X,
                     int kcmax, int nmember) {
  const dim3 g(std::max(1, l.grid / std::max(1, kcmax)), kcmax);
  k_mom_flux<<<g, NT, 0, l.stream>>>(S, M, l.ntile);
  k_mom_accel<<<g, NT, 0, l.stream>>>(S, M, l.ntile);
  k_mom_edges<<<nmember, 64, 0, l.stream>>>(S, M);
  k_mom_sum<<<l.grid, NT, 0, l.stream>>>(S, M, X, l.ntile);
  count_launches(4);
}

}  // namespace xm
