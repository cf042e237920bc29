// xm_kernels.h -- launch interface between the host orchestration (xm_capi.cu)
// and the kernel files (xm_step.cu FP64, xm_mixed.cu FP32 inner solve).
#pragma once

#include <algorithm>

#include "../../include/efdc_xm.h"
#include "xm_internal.h"

namespace xm {

struct Launch {
  int grid;          // CTAs of the grid-stride cell kernels (one tile per CTA pass)
  int grid_cg;       // CTAs of the FP64 CG kernels (one quad of 4 tiles per CTA pass)
  int grid_cg32;     // CTAs of the FP32 matrix-vector kernel
  int grid_up32;     // CTAs of the FP32 update kernel
  int ntile;         // tiles including the ghost tile 0
  int nsm;           // SMs of the device
  cudaStream_t stream;
  bool mx_jac = true;    // MIXED: some member runs the Jacobi inner solve
  bool mx_poly = false;  // MIXED: some member runs the polynomial-preconditioned one
  bool may_asym = true;  // some member's operator can be unsymmetric (else symmetric kernels)
  bool chan = false;     // sub-grid channel terms (a step of a context with channels)
  bool baro = false;     // some member of the step has the baroclinic terms (CALEBI)
  // schedule (efdc_xm_set_schedule): the FP32 CG kernels' variant (0: quad
  // descriptors prefetched one quad ahead, 1: in shared-memory batches) and,
  // for variant 1, caps on their resident CTAs per SM (0: occupancy)
  int variant = 0;
  int ctas_mv = 0, ctas_up = 0;
  // MIXED: the inner solve's target is the reduction the FP64 residual needs
  // to reach its stop, times this margin (< 1 over-solves the FP32 inner
  // solve so that fewer refinement passes are needed)
  double inner_margin = 1.0;
  // the member reductions folded into the CG kernels (no member-reduce
  // kernels); off where sub-grid channel kernels add to the partials
  bool fold = false;
};

// One array to move between host order and tile order (see k_scatter).
struct CopyJob {
  const void *host_order;  // device staging buffer: every member's array back to back
  void *dev;               // tile-order device array
  int is_int;              // 0 double, 1 LOGICAL (0/1), 2 raw int, 3 double water-only
};

// copy: the two-level advance as per-cell copies (a subset of the members
// steps), else the host has swapped the buffers
void launch_begin(const Launch &l, const DevStatic &S, const DevState &X, const int *act,
                  bool copy);
// CALPUV9C: the kernels up to the time-level advance, and the copies of the advance
void launch_begin3(const Launch &l, const DevStatic &S, const DevState &X, const int *act);
void launch_advance3(const Launch &l, const DevStatic &S, const DevState &X);
// CALEXP2T's external-mode terms of every member with its static part; the
// depth sums go to X.fcaxe, X.fcaye, X.fxe, X.fye.
void launch_explicit(const Launch &l, const DevStatic &S, const MomDev &M, const DevState &X,
                     int kcmax, int nmember);
// the implicit bottom / vegetation drag (RCX, RCY) of the members with ISITB >= 1
// or ISVEG > 0, after the begin kernel
void launch_implicit_drag(const Launch &l, const DevStatic &S, const DevState &X,
                          const int *act);
void launch_put(cudaStream_t st, const int *idx, const double *val, int n, double *dst);
// CONGRAD of small members, one CTA each with its vectors in shared memory
// (k_cg_small): the windows of every member fit when cg_small_fits(the
// largest window's slots); the same iterates as the multi-kernel CG.
constexpr int SMALL_SMEM_MAX = 200 * 1024;
bool cg_small_fits(int slots);
void launch_cg_small(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P,
                     Ctl *ctl, Glob *glob, double *part, int max_slots, int max_units,
                     int nmember);
void launch_put_int(cudaStream_t st, const int *idx, const int *val, int n, int *dst);
// sub-grid channels (xm_chan.cu); each does nothing unless l.chan
void launch_chan_entry(const Launch &l, const DevStatic &S, const DevState &X, const int *act);
void launch_chan_sub(const Launch &l, const DevStatic &S, const DevState &X, Ctl *ctl,
                     const int *act, int first_sweep);
void launch_chan_res64(const Launch &l, const DevStatic &S, const DevSystem &Y, const double *P,
                       const Ctl *ctl, double *part);
void launch_chan_mv64(const Launch &l, const DevStatic &S, const DevSystem &Y, const Ctl *ctl,
                      double *part);
void launch_chan_flow(const Launch &l, const DevStatic &S, const DevState &X, const int *act);
void launch_chan_exch(const Launch &l, const DevStatic &S, const DevState &X, const int *act);
void launch_chan_p0(const Launch &l, const DevStatic &S, const SysView &V, const double *P,
                    const int *act);
void launch_chan_resmx(const Launch &l, const DevStatic &S, const SysView &V, const DevSystem &Y,
                       const double *P, const Ctl *ctl, double *part);
void launch_chan_mvmx(const Launch &l, const DevStatic &S, const DevSystem &Y, const Ctl *ctl,
                      double *part);
void launch_sweep_reset(const Launch &l, Ctl *ctl, const int *act, int nmember);
void launch_assemble(const Launch &l, const DevStatic &S, const DevState &X, Ctl *ctl,
                     const int *act);
void launch_obc(const Launch &l, const DevStatic &S, const DevState &X, const DevObc &B, Ctl *ctl,
                const int *act, bool serial, int write_cross);
void launch_obc_reset(const Launch &l, const DevStatic &S, const DevObc &B, const DevState &X,
                      const int *act);
void launch_scale(const Launch &l, const DevStatic &S, const DevState &X, const DevSystem &Y,
                  Ctl *ctl, const int *act, int mixed, int write_cross);
void launch_solve_reset(const Launch &l, Ctl *ctl, Glob *glob, const int *act, int nmember);
void launch_outer_reset(const Launch &l, Glob *glob);
void launch_cg_init(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P, Ctl *ctl,
                    Glob *glob, double *part);
void launch_cg_iter(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P, Ctl *ctl,
                    Glob *glob, double *part);
void launch_cg_matvec(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P,
                      Ctl *ctl, double *part);
void launch_cg_update(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      Glob *glob, double *part, int no_stop);
// after the FP64 CG loop: the last iteration's P += alpha*p of every member
// that iterated (each matrix-vector kernel adds the previous iteration's)
void launch_cg_finish(const Launch &l, const DevStatic &S, const DevSystem &Y, double *P,
                      const Ctl *ctl);
void launch_mx_resid(const Launch &l, const DevStatic &S, const SysView &V, const DevSystem &Y,
                     const double *P, Ctl *ctl, Glob *glob, double *part, double rsqm_fac,
                     double rel_tol, int no_stop);
void launch_mx_apply(const Launch &l, const DevStatic &S, const SysView &V, const DevSystem &Y,
                     double *P, const Ctl *ctl);
void launch_mx_matvec(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      double *part);
void launch_mx_update(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      Glob *glob, double *part, int no_stop);
void launch_mx_zinit(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                     double *part);
void launch_mx_iter(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl, Glob *glob,
                    double *part);
void launch_backsub(const Launch &l, const DevStatic &S, const DevState &X, const int *act);
void launch_obc_hp(const Launch &l, const DevStatic &S, const DevState &X, const DevObc &B,
                   const int *act);
void launch_wetdry(const Launch &l, const DevStatic &S, const DevState &X, Ctl *ctl,
                   const int *act, bool any_legacy, bool any99);
void launch_final(const Launch &l, const DevStatic &S, const DevState &X, Ctl *ctl,
                  const int *act, bool any_waste);
void launch_reciprocals(const Launch &l, const DevStatic &S, const DevState &X, int t0, int t1);
// the autotuner's initial guess of a timed solve: P at the last step's entry
void launch_tune_guess(const Launch &l, const DevStatic &S, const DevState &X, double *out);
// the bed's derived arrays (ZBRATU, ZBRATV, SGZUU, SGZVV) of the tiles [t0, t1)
void launch_bed(cudaStream_t st, const DevStatic &S, const DevBed &Bd, const double *dxp,
                const double *dyp, const double *dzc1, const double *sgzu1, const double *sgzv1,
                double gu, double gv, int t0, int t1);
// the bottom-stress producer (CALTBXY + TBX/TBY) of the members with ds[m].on
void launch_tbxy(const Launch &l, const DevStatic &S, const DevState &X, const DevBed &Bd,
                 const DragScalars *ds);
// copies `bytes` (a multiple of 4) from src to dst, or zeros dst when src is
// null, with a kernel (either side may be mapped pinned host memory)
void launch_words(cudaStream_t st, void *dst, const void *src, size_t bytes);
// slots [d0, d1)
void launch_scatter(cudaStream_t st, const CopyJob *jobs, int njob, const int *lidx,
                    const int *tile_member, const long long *moff, const int *mlc, int d0,
                    int d1);
void launch_gather(cudaStream_t st, const CopyJob *jobs, int njob, const int *lidx,
                   const int *tile_member, const long long *moff, int d0, int d1);
void launch_sys_prepare(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                        int mixed);

// calibration: drag from log n, and the reverse of one step (xm_adjoint.cu)
void launch_cal_tbxy(const Launch &l, const DevStatic &S, const DevState &X, const DevCalib &A);
void launch_adj_gauge(const Launch &l, const int *slots, const double *w, int n, double *ap);
void launch_adj_pre(const Launch &l, const DevStatic &S, const DevState &X, const DevObc &B,
                    const DevCalib &A);
void launch_adj_rhs(const Launch &l, const DevStatic &S, const DevSystem &Y, const Ctl *ctl,
                    const DevCalib &A, double *bsq);
void launch_adj_post(const Launch &l, const DevStatic &S, const DevState &X, const DevObc &B,
                     const DevCalib &A);
void launch_gather_slots(cudaStream_t st, const double *src, const int *slots, int n, double *out);

// loop control of a step that runs as one graph (xm_loop.cu): each loop is a
// conditional WHILE node whose handle these kernels set
void launch_loop_enter(cudaStream_t st, Glob *g, int which, cudaGraphConditionalHandle h,
                       int pending, int nmember);
void launch_loop_next(cudaStream_t st, Glob *g, int which, cudaGraphConditionalHandle h, int cap,
                      int inner, int nmember);
void launch_step_enter(cudaStream_t st, Ctl *ctl, const int *act, Glob *g, int nmember);
void launch_inner_done(cudaStream_t st, Ctl *ctl, const int *act, int nmember);
void launch_after_solve(cudaStream_t st, Ctl *ctl, int *act, int nmember, int mixed);
void launch_sweep_next(cudaStream_t st, const DevStatic &S, Ctl *ctl, int *act, Glob *g,
                       cudaGraphConditionalHandle h, int cap, int nmember);
void launch_fin_prepare(cudaStream_t st, const Ctl *ctl, int *act, int nmember);

// sets the message returned by efdc_xm_last_error() for this thread
void set_last_error_str(const char *msg);

// process-wide count of kernel launches (measurement hook)
void count_launches(int n);

int occupancy_blocks_per_sm();
int occupancy_blocks_per_sm_cg();
int occupancy_blocks_per_sm_mixed();
int occupancy_blocks_per_sm_mixed_update();

}  // namespace xm
