// xm_mixed.cu -- FP32 inner preconditioned CG of the MIXED form.
//
// The correction system (the Jacobi-scaled operator Ahat = D^-1/2 A D^-1/2,
// unit diagonal, rhs = the FP64 refinement residual scaled and rounded to
// FP32) is solved by preconditioned CG with FP32 operator, vectors and axpys
// and FP64 dot products (per thread, per quad and in the fixed-order member
// sums).  The preconditioner is the two-term Neumann series of Ahat^-1,
// z = (2I - Ahat) r: about half the iterations of plain Jacobi-PCG
// (congrad.f90:91-169) for one extra stencil on r per iteration, folded into
// the update kernel.  Well-conditioned members (few Jacobi iterations) keep
// plain Jacobi, whose iteration is cheaper; the host chooses per member.
// The outer FP64 loop (xm_step.cu: k_mx_resid / k_mx_apply) keeps P in FP64
// and stops on the reference's own criterion, the FP64 RSQ <= RSQM.

#include "xm_cg.cuh"
#include "xm_kernels.h"

namespace xm {

#define TILE_LOOP(ntile)                                                      \
  for (int tile = blockIdx.x + 1; tile < (ntile); tile += gridDim.x)

// p = z + beta*p_old at the cell and its halo (z = r for Jacobi members),
// Ahat*p, p.Ap (per member).
template <bool MA>
__global__ void __launch_bounds__(NT, 6) k_mx_matvec(DevStatic S, DevSystem Y, const Ctl *ctl,
                                                    double *part) {
  struct A {
    bool skip, asym;
    float beta;
    const float *pold;
    float *pnew;
    const float *z;
  };
  quad_sweep<1>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        const bool asym = unsym<MA>(k);
        const bool poly = Y.mpoly[m] && !asym;
        return A{(k.done | k.idone) != 0, asym, float(k.beta), par ? Y.pb32 : Y.pa32,
                 par ? Y.pa32 : Y.pb32, poly ? Y.z32 : (par ? Y.r32b : Y.r32)};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        v[0] = matvec_row_scaled(g, valid, a.z, a.pold, a.pnew, Y.as32, Y.aw32, Y.ae32, Y.an32,
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

// x += alpha*p, r -= alpha*Ap, z = (2I - Ahat) r (the two-term Neumann
// polynomial), r.z and r.r (FP64 sums): the members that use it.
__global__ void __launch_bounds__(NT, 6) k_mx_update_poly(DevStatic S, DevSystem Y,
                                                         const Ctl *ctl, double *part) {
  struct A {
    bool skip;
    float alpha;
    const float *pnew;
    const float *r;
    float *rnew;
  };
  quad_sweep<2>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        const bool poly = Y.mpoly[m] && !unsym<true>(k);
        return A{(k.done | k.idone) != 0 || !poly, float(k.alpha), par ? Y.pa32 : Y.pb32,
                 par ? Y.r32b : Y.r32, par ? Y.r32 : Y.r32b};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        update_row_poly(g, valid, Y.x32, a.pnew, a.r, a.rnew, Y.ap32, Y.as32, Y.aw32, Y.z32,
                        a.alpha, true, v[0], v[1]);
      });
}
// The same for the Jacobi members (z = r): x, r and r.r only.
__global__ void __launch_bounds__(NT) k_mx_update_jac(DevStatic S, DevSystem Y, const Ctl *ctl,
                                                     double *part) {
  struct A {
    bool skip;
    float alpha;
    const float *pnew;
    const float *r;
    float *rnew;
  };
  quad_sweep<2>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        const bool poly = Y.mpoly[m] && !unsym<true>(k);
        return A{(k.done | k.idone) != 0 || poly, float(k.alpha), par ? Y.pa32 : Y.pb32,
                 par ? Y.r32b : Y.r32, par ? Y.r32 : Y.r32b};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        double rr = 0.0;
        update_row_jac(g, valid, Y.x32, a.pnew, a.r, a.rnew, Y.ap32, a.alpha, rr);
        v[0] = rr;
        v[1] = rr;
      });
}
// BETA = r.z / r.z_old and the inner stop test on r.r.  With no_stop the
// inner solve runs past its target (kernel timing only).
__global__ void __launch_bounds__(NT) k_red_mx_update(DevStatic S, Ctl *ctl, Glob *glob,
                                                     const double *part, double total_cap_fac,
                                                     int no_stop) {
  member_reduce<2>(
      S, part, [&](int m) { return (ctl[m].done | ctl[m].idone) != 0; },
      [&](int m, const double *sum) {
        if (threadIdx.x != 0) return;
        Ctl &k = ctl[m];
        const double rz = sum[0], rr = sum[1];
        const int iterm = S.sc[m].iterm;
        k.beta = rz / k.rpcg;
        k.rpcg = rz;
        k.rsq = rr;
        const int it = k.inner_iter + 1;
        k.inner_iter = it;
        k.iter += 1;
        if (!isfinite(rr) || !isfinite(rz) || !isfinite(k.alpha)) {
          k.status = EFDC_XM_NONFINITE;
          k.done = 1;
          atomicAdd(&glob->ndone, 1);
        } else if (!no_stop && (rr <= k.rsq_target || it >= iterm ||
                                k.iter >= int(total_cap_fac * iterm) + 50)) {
          k.idone = 1;
          atomicAdd(&glob->nidone, 1);
        } else {
          k.parity ^= 1;
        }
      });
}

// First inner iteration of the polynomial members: z0 = (2I - Ahat) r0,
// p_old = 0, RPCG = r0.z0 (Jacobi members start from k_mx_resid's p0 = r0).
__global__ void __launch_bounds__(NT) k_mx_zinit(DevStatic S, DevSystem Y, const Ctl *ctl,
                                                double *part) {
  struct A {
    bool skip, asym;
  };
  quad_sweep<1>(
      S, part,
      [&](int m) { return A{ctl[m].done != 0 || !Y.mpoly[m] || unsym<true>(ctl[m]), false}; },
      [&](const A &, const RowGeo &g, bool valid, double *v) {
        v[0] = zinit_row(g, valid, Y.r32, Y.as32, Y.aw32, Y.z32, Y.pa32, true);
      });
}
__global__ void __launch_bounds__(NT) k_red_mx_zinit(DevStatic S, DevSystem Y, Ctl *ctl,
                                                     const double *part) {
  member_reduce<1>(
      S, part, [&](int m) { return ctl[m].done != 0 || !Y.mpoly[m] || unsym<true>(ctl[m]); },
      [&](int m, const double *sum) {
        if (threadIdx.x == 0) ctl[m].rpcg = sum[0];
      });
}

static int reduce_grid(const DevStatic &S) { return std::min(S.nmember, 1024); }

void launch_mx_matvec(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      double *part) {
  if (l.may_asym)
    k_mx_matvec<true><<<l.grid_cg32, NT, 0, l.stream>>>(S, Y, ctl, part);
  else
    k_mx_matvec<false><<<l.grid_cg32, NT, 0, l.stream>>>(S, Y, ctl, part);
  launch_chan_mvmx(l, S, Y, ctl, part);
  k_red_mx_matvec<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, part);
  count_launches(2);
}
void launch_mx_update(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      Glob *glob, double *part, int no_stop) {
  if (l.mx_jac) {
    k_mx_update_jac<<<l.grid_up32, NT, 0, l.stream>>>(S, Y, ctl, part);
    count_launches(1);
  }
  if (l.mx_poly) {
    k_mx_update_poly<<<l.grid_up32, NT, 0, l.stream>>>(S, Y, ctl, part);
    count_launches(1);
  }
  k_red_mx_update<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, glob, part, 2.0, no_stop);
  count_launches(1);
}
void launch_mx_zinit(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                     double *part) {
  if (!l.mx_poly) return;
  k_mx_zinit<<<l.grid_up32, NT, 0, l.stream>>>(S, Y, ctl, part);
  k_red_mx_zinit<<<reduce_grid(S), NT, 0, l.stream>>>(S, Y, ctl, part);
  count_launches(2);
}
void launch_mx_iter(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl, Glob *glob,
                    double *part) {
  launch_mx_matvec(l, S, Y, ctl, part);
  launch_mx_update(l, S, Y, ctl, glob, part, 0);
}

int occupancy_blocks_per_sm_mixed_update() {
  int b = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_mx_update_poly, NT, 0);
  return b > 0 ? b : 1;
}

int occupancy_blocks_per_sm_mixed() {
  int a = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_mx_matvec<true>, NT, 0);
  return a > 0 ? a : 1;
}

}  // namespace xm
