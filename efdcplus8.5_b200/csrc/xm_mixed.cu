// xm_mixed.cu -- FP32 inner preconditioned CG of the MIXED form.
//
// The correction system A*x = r (r = FP64 refinement residual rounded to
// FP32) is solved with the same Jacobi-PCG as CONGRAD (congrad.f90:91-169),
// but the operator, the vectors and the axpys are FP32; the dot products are
// accumulated in FP64 (per thread, per CTA and in the fixed-order final sum).
// The outer FP64 loop (xm_step.cu: k_mx_resid / k_mx_apply) keeps P in FP64
// and stops on the reference's own criterion, the FP64 RSQ <= RSQM.

#include "xm_cg.cuh"
#include "xm_kernels.h"

namespace xm {

#define TILE_LOOP(ntile)                                                      \
  for (int tile = blockIdx.x + 1; tile < (ntile); tile += gridDim.x)

// p = z + beta*p_old at the cell and its neighbours, Ap, p.Ap, ALPHA.
__global__ void __launch_bounds__(NT, 5) k_mx_matvec(DevStatic S, DevSystem Y, int ntile, Ctl *ctl,
                                                 double *part) {
  __shared__ double sh[32];
  if (ctl->done | ctl->idone) return;
  const float beta = float(ctl->beta);
  const bool par = ctl->parity;
  const float *pold = par ? Y.pb32 : Y.pa32;
  float *pnew = par ? Y.pa32 : Y.pb32;
  const bool asym = ctl->asym;
  double acc = 0.0;
  CG_TILE_LOOP(ntile) {
    CG_TILE_GEO(S);
    acc += matvec_row_scaled(g, valid, Y.r32, pold, pnew, Y.as32, Y.aw32, Y.ae32, Y.an32, Y.ap32,
                             beta, asym);
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
  if (arrive_last(&ctl->counter)) {
    const double papcg = reduce_partials(part, gridDim.x, sh);
    if (threadIdx.x == 0) {
      ctl->papcg = papcg;
      ctl->alpha = ctl->rpcg / papcg;
      ctl->counter = 0;
    }
  }
}

// x += alpha*p, r -= alpha*Ap, r.z and r.r (FP64 sums), BETA, inner stop test.
__global__ void __launch_bounds__(NT) k_mx_update(DevStatic S, DevSystem Y, int ntile, Ctl *ctl,
                                                 double *part, int inner_cap, int total_cap) {
  __shared__ double sh[32];
  if (ctl->done | ctl->idone) return;
  const float alpha = float(ctl->alpha);
  const float *pnew = ctl->parity ? Y.pa32 : Y.pb32;
  double a1 = 0.0;
  CG_TILE_LOOP(ntile) {
    CG_TILE_GEO(S);
    update_row_scaled(g, valid, Y.x32, pnew, Y.r32, Y.ap32, alpha, a1);
  }
  a1 = block_sum(a1, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = a1;
  if (arrive_last(&ctl->counter)) {
    const double rz = reduce_partials(part, gridDim.x, sh);  // r.z = r.r (unit diagonal)
    const double rr = rz;
    if (threadIdx.x == 0) {
      ctl->beta = rz / ctl->rpcg;
      ctl->rpcg = rz;
      ctl->rsq = rr;
      const int it = ctl->inner_iter + 1;
      ctl->inner_iter = it;
      ctl->iter += 1;
      if (!isfinite(rr) || !isfinite(ctl->alpha)) {
        ctl->done = 1;
        ctl->status = EFDC_XM_NONFINITE;
      } else if (rr <= ctl->rsq_target || it >= inner_cap || ctl->iter >= total_cap) {
        ctl->idone = 1;
      } else {
        ctl->parity ^= 1;
      }
      ctl->counter = 0;
    }
  }
}

void launch_mx_matvec(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      double *part) {
  k_mx_matvec<<<l.grid_cg32, NT, 0, l.stream>>>(S, Y, l.ntile, ctl, part);
  count_launches(1);
}
void launch_mx_update(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      double *part, int inner_cap, int total_cap) {
  k_mx_update<<<l.grid_up32, NT, 0, l.stream>>>(S, Y, l.ntile, ctl, part, inner_cap, total_cap);
  count_launches(1);
}
void launch_mx_iter(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                    double *part, int inner_cap, int total_cap) {
  k_mx_matvec<<<l.grid_cg32, NT, 0, l.stream>>>(S, Y, l.ntile, ctl, part);
  count_launches(1);
  k_mx_update<<<l.grid_up32, NT, 0, l.stream>>>(S, Y, l.ntile, ctl, part, inner_cap, total_cap);
  count_launches(1);
}

int occupancy_blocks_per_sm_mixed_update() {
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_mx_update, NT, 0);
  return b > 0 ? b : 1;
}

int occupancy_blocks_per_sm_mixed() {
  int a = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_mx_matvec, NT, 0);
  return a > 0 ? a : 1;
}

}  // namespace xm
