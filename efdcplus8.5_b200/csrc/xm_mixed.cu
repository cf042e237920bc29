// xm_mixed.cu -- FP32 inner preconditioned CG of the MIXED form.
//
// The correction system A*x = r (r = FP64 refinement residual rounded to
// FP32) is solved with the same Jacobi-PCG as CONGRAD (congrad.f90:91-169),
// but the operator, the vectors and the axpys are FP32; the dot products are
// accumulated in FP64 (per thread, per CTA and in the fixed-order final sum).
// The outer FP64 loop (xm_step.cu: k_mx_resid / k_mx_apply) keeps P in FP64
// and stops on the reference's own criterion, the FP64 RSQ <= RSQM.

#include "xm_common.cuh"
#include "xm_kernels.h"

namespace xm {

#define TILE_LOOP(ntile)                                                      \
  for (int tile = blockIdx.x + 1; tile < (ntile); tile += gridDim.x)

__device__ __forceinline__ float rcpf(float x) { return __frcp_rn(x); }

// p = z + beta*p_old at the cell and its neighbours, Ap, p.Ap, ALPHA.
__global__ void __launch_bounds__(NT) k_mx_matvec(DevStatic S, DevSystem Y, int ntile, Ctl *ctl,
                                                 double *part) {
  __shared__ double sh[32];
  if (ctl->done | ctl->idone) return;
  const float beta = float(ctl->beta);
  const bool par = ctl->parity;
  const float *__restrict__ pold = par ? Y.pb32 : Y.pa32;
  float *__restrict__ pnew = par ? Y.pa32 : Y.pb32;
  const bool asym = ctl->asym;
  const float *__restrict__ r = Y.r32;
  const float *__restrict__ ccc = Y.ccc32;
  double acc = 0.0;
  TILE_LOOP(ntile) {
    const Nb q = neighbours(S.tnbr, tile, threadIdx.x);
    const int d = q.d;
    if (S.kind[d] == LAND) continue;
    auto pc = [&](int j) { return fmaf(beta, pold[j], r[j] * rcpf(ccc[j])); };
    const float p = pc(d), pn = pc(q.n), pe = pc(q.e), pw = pc(q.w), ps = pc(q.s);
    float ccn, cce;
    if (asym) {
      ccn = Y.ccn32[d];
      cce = Y.cce32[d];
    } else {
      ccn = Y.ccs32[q.n];
      cce = Y.ccw32[q.e];
    }
    const float ap = ccc[d] * p + Y.ccs32[d] * ps + ccn * pn + Y.ccw32[d] * pw + cce * pe;
    pnew[d] = p;
    Y.ap32[d] = ap;
    acc += double(ap) * double(p);
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
  const float *__restrict__ pnew = ctl->parity ? Y.pa32 : Y.pb32;
  double a1 = 0.0, a2 = 0.0;
  TILE_LOOP(ntile) {
    const int d = tile * TILE + threadIdx.x;
    if (S.kind[d] == LAND) continue;
    Y.x32[d] = fmaf(alpha, pnew[d], Y.x32[d]);
    const float r = fmaf(-alpha, Y.ap32[d], Y.r32[d]);
    Y.r32[d] = r;
    const float z = r * rcpf(Y.ccc32[d]);
    a1 += double(r) * double(z);
    a2 += double(r) * double(r);
  }
  a1 = block_sum(a1, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = a1;
  a2 = block_sum(a2, sh);
  if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = a2;
  if (arrive_last(&ctl->counter)) {
    const double rz = reduce_partials(part, gridDim.x, sh);
    const double rr = reduce_partials(part + gridDim.x, gridDim.x, sh);
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
  k_mx_matvec<<<l.grid, NT, 0, l.stream>>>(S, Y, l.ntile, ctl, part);
  count_launches(1);
}
void launch_mx_update(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      double *part, int inner_cap, int total_cap) {
  k_mx_update<<<l.grid, NT, 0, l.stream>>>(S, Y, l.ntile, ctl, part, inner_cap, total_cap);
  count_launches(1);
}
void launch_mx_iter(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                    double *part, int inner_cap, int total_cap) {
  k_mx_matvec<<<l.grid, NT, 0, l.stream>>>(S, Y, l.ntile, ctl, part);
  count_launches(1);
  k_mx_update<<<l.grid, NT, 0, l.stream>>>(S, Y, l.ntile, ctl, part, inner_cap, total_cap);
  count_launches(1);
}

int occupancy_blocks_per_sm_mixed() {
  int a = 0, b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_mx_matvec, NT, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_mx_update, NT, 0);
  const int m = std::min(a, b);
  return m > 0 ? m : 1;
}

}  // namespace xm
