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

// p = r + beta*p_old at the cell and its halo, Ahat*p, p.Ap (per member).
__global__ void __launch_bounds__(NT, 5) k_mx_matvec(DevStatic S, DevSystem Y, const Ctl *ctl,
                                                    double *part) {
  struct A {
    bool skip, asym;
    float beta;
    const float *pold;
    float *pnew;
  };
  quad_sweep<1>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        return A{(k.done | k.idone) != 0, k.asym != 0, float(k.beta), par ? Y.pb32 : Y.pa32,
                 par ? Y.pa32 : Y.pb32};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        v[0] = matvec_row_scaled(g, valid, Y.r32, a.pold, a.pnew, Y.as32, Y.aw32, Y.ae32, Y.an32,
                                 Y.ap32, a.beta, a.asym);
      });
}
// ALPHA = RPCG / p.Ap
__global__ void __launch_bounds__(NT) k_red_mx_matvec(DevStatic S, Ctl *ctl, const double *part) {
  member_reduce<1>(
      S, part, [&](int m) { return (ctl[m].done | ctl[m].idone) != 0; },
      [&](int m, const double *sum) {
        if (threadIdx.x != 0) return;
        ctl[m].papcg = sum[0];
        ctl[m].alpha = ctl[m].rpcg / sum[0];
      });
}

// x += alpha*p, r -= alpha*Ap, r.r (FP64 sums; = r.z on the unit-diagonal
// system).
__global__ void __launch_bounds__(NT) k_mx_update(DevStatic S, DevSystem Y, const Ctl *ctl,
                                                 double *part) {
  struct A {
    bool skip;
    float alpha;
    const float *pnew;
  };
  quad_sweep<1>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        return A{(k.done | k.idone) != 0, float(k.alpha), k.parity ? Y.pa32 : Y.pb32};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        update_row_scaled(g, valid, Y.x32, a.pnew, Y.r32, Y.ap32, a.alpha, v[0]);
      });
}
// BETA and the inner stop test.  With no_stop the inner solve runs past its
// target (kernel timing only).
__global__ void __launch_bounds__(NT) k_red_mx_update(DevStatic S, Ctl *ctl, Glob *glob,
                                                     const double *part, double total_cap_fac,
                                                     int no_stop) {
  member_reduce<1>(
      S, part, [&](int m) { return (ctl[m].done | ctl[m].idone) != 0; },
      [&](int m, const double *sum) {
        if (threadIdx.x != 0) return;
        Ctl &k = ctl[m];
        const double rz = sum[0];
        const int iterm = S.sc[m].iterm;
        k.beta = rz / k.rpcg;
        k.rpcg = rz;
        k.rsq = rz;
        const int it = k.inner_iter + 1;
        k.inner_iter = it;
        k.iter += 1;
        if (!isfinite(rz) || !isfinite(k.alpha)) {
          k.status = EFDC_XM_NONFINITE;
          k.done = 1;
          atomicAdd(&glob->ndone, 1);
        } else if (!no_stop && (rz <= k.rsq_target || it >= iterm ||
                                k.iter >= int(total_cap_fac * iterm) + 50)) {
          k.idone = 1;
          atomicAdd(&glob->nidone, 1);
        } else {
          k.parity ^= 1;
        }
      });
}

static int reduce_grid(const DevStatic &S) { return std::min(S.nmember, 1024); }

void launch_mx_matvec(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      double *part) {
  k_mx_matvec<<<l.grid_cg32, NT, 0, l.stream>>>(S, Y, ctl, part);
  k_red_mx_matvec<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, part);
  count_launches(2);
}
void launch_mx_update(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      Glob *glob, double *part, int no_stop) {
  k_mx_update<<<l.grid_up32, NT, 0, l.stream>>>(S, Y, ctl, part);
  k_red_mx_update<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, glob, part, 2.0, no_stop);
  count_launches(2);
}
void launch_mx_iter(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl, Glob *glob,
                    double *part) {
  launch_mx_matvec(l, S, Y, ctl, part);
  launch_mx_update(l, S, Y, ctl, glob, part, 0);
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
