// xm_loop.cu -- loop control of a step that runs as one CUDA graph.
//
// The reference's step has three loops whose exit is data-dependent: the CG
// iterations (congrad.f90:91-169, stop at RSQ <= RSQM or ITERM), the MIXED
// form's refinement passes around its FP32 inner iterations, and the wet/dry
// re-solves (GOTO 1000 at calpuv2c.f90:597-601 and :726-749, at most
// NCORDRY = 500).  In a device-driven step each loop is a conditional WHILE
// node of the step's graph, and the small kernels below decide, on the
// device, whether its body runs again: from the member counters the reduce
// kernels keep (Glob::ndone, Glob::nidone) and a body counter with a fixed
// cap, so that every loop ends even if a counter were wrong.  The per-member
// bookkeeping the host did between sweeps (stats, failed members leaving the
// step, the sweep count and its cap) is done here too, so a step needs no
// host synchronisation until it has finished.

#include "xm_kernels.h"

namespace xm {

// Start of a loop: its body counter to 0 and the condition of its first
// body: 1, or (pending) "some member has not finished its solve".
__global__ void k_loop_enter(Glob *g, int which, cudaGraphConditionalHandle h, int pending,
                             int nmember) {
  g->loop[which] = 0;
  cudaGraphSetConditional(h, (!pending || g->ndone < nmember) ? 1u : 0u);
}

// End of a loop body: count it and decide on the next.  inner: the MIXED inner
// loop, which runs while some member's inner solve is unfinished.
__global__ void k_loop_next(Glob *g, int which, cudaGraphConditionalHandle h, int cap, int inner,
                            int nmember) {
  g->tot[which] += 1;
  const int c = ++g->loop[which];
  const bool more = inner ? (g->nidone + g->ndone < nmember) : (g->ndone < nmember);
  cudaGraphSetConditional(h, (more && c < cap) ? 1u : 0u);
}

// Start of a step: the members taking part, the step counters of Glob.
__global__ void k_step_enter(Ctl *ctl, const int *act, Glob *g, int nmember) {
  for (int m = threadIdx.x; m < nmember; m += blockDim.x) ctl[m].stepping = act[m] ? 1 : 0;
  if (threadIdx.x < NLOOP) g->tot[threadIdx.x] = 0;
}

// MIXED, after an inner loop: the inner iterations of the pass (those of the
// first pass choose the next step's inner preconditioner).
__global__ void k_inner_done(Ctl *ctl, const int *act, int nmember) {
  for (int m = threadIdx.x; m < nmember; m += blockDim.x) {
    Ctl &k = ctl[m];
    if (!act[m] || k.inner_iter <= 0) continue;
    k.last_inner = k.inner_iter;
    if (k.outer == 1) k.inner_first = k.inner_iter;
  }
}

// After a solve: the member's statistics, and a member whose solve failed
// leaves the step before its back-substitution (its status is kept).
__global__ void k_after_solve(Ctl *ctl, int *act, int nmember, int mixed) {
  for (int m = threadIdx.x; m < nmember; m += blockDim.x) {
    if (!act[m]) continue;
    Ctl &k = ctl[m];
    k.iters_last = k.iter;
    k.iters_total += k.iter;
    k.solves += 1;
    k.rsq_last = mixed ? k.rsq64 : k.rsq;
    k.outer_total += k.outer;
    k.ccmnm_last = fmin(k.ccmnm_int, k.ccmnm_bc);
    if (!k.done && k.status == 0) k.status = EFDC_XM_CG_MAXITER;
    int st = EFDC_XM_OK;
    if (k.asym & 2)
      st = EFDC_XM_UNSUPPORTED;
    else if (k.status != EFDC_XM_OK)
      st = k.status;
    if (st != EFDC_XM_OK) {
      k.mstatus = st;
      act[m] = 0;
    }
  }
}

// End of a sweep (calpuv2c.f90:597-601, 726-749): a member whose faces
// changed sweeps again unless it has reached its cap (then its status is
// WETDRY_MAXSWEEP); the sweep loop runs again while some member does.
__global__ void k_sweep_next(DevStatic S, Ctl *ctl, int *act, Glob *g,
                             cudaGraphConditionalHandle h, int cap, int nmember) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int m = threadIdx.x; m < nmember; m += blockDim.x) {
    if (!act[m]) continue;
    Ctl &k = ctl[m];
    const StepScalars &c = S.sc[m];
    int next = 0;
    if (c.isdry > 0 && c.isdry != 98 && k.icordry) {
      if (++k.sweep < c.max_sweeps)
        next = 1;
      else
        k.mstatus = EFDC_XM_WETDRY_MAXSWEEP;
    }
    act[m] = next;
    if (next) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    g->tot[LOOP_SWEEP] += 1;
    const int c = ++g->loop[LOOP_SWEEP];
    cudaGraphSetConditional(h, (any && c < cap) ? 1u : 0u);
  }
}

// Before the finalisation: the members whose sweeps ended normally.
__global__ void k_fin_prepare(const Ctl *ctl, int *act, int nmember) {
  for (int m = threadIdx.x; m < nmember; m += blockDim.x)
    act[m] = (ctl[m].stepping && ctl[m].mstatus == EFDC_XM_OK) ? 1 : 0;
}

void launch_loop_enter(cudaStream_t st, Glob *g, int which, cudaGraphConditionalHandle h,
                       int pending, int nmember) {
  k_loop_enter<<<1, 1, 0, st>>>(g, which, h, pending, nmember);
  count_launches(1);
}
void launch_loop_next(cudaStream_t st, Glob *g, int which, cudaGraphConditionalHandle h, int cap,
                      int inner, int nmember) {
  k_loop_next<<<1, 1, 0, st>>>(g, which, h, cap, inner, nmember);
  count_launches(1);
}
void launch_step_enter(cudaStream_t st, Ctl *ctl, const int *act, Glob *g, int nmember) {
  k_step_enter<<<1, 256, 0, st>>>(ctl, act, g, nmember);
  count_launches(1);
}
void launch_inner_done(cudaStream_t st, Ctl *ctl, const int *act, int nmember) {
  k_inner_done<<<1, 256, 0, st>>>(ctl, act, nmember);
  count_launches(1);
}
void launch_after_solve(cudaStream_t st, Ctl *ctl, int *act, int nmember, int mixed) {
  k_after_solve<<<1, 256, 0, st>>>(ctl, act, nmember, mixed);
  count_launches(1);
}
void launch_sweep_next(cudaStream_t st, const DevStatic &S, Ctl *ctl, int *act, Glob *g,
                       cudaGraphConditionalHandle h, int cap, int nmember) {
  k_sweep_next<<<1, 256, 0, st>>>(S, ctl, act, g, h, cap, nmember);
  count_launches(1);
}
void launch_fin_prepare(cudaStream_t st, const Ctl *ctl, int *act, int nmember) {
  k_fin_prepare<<<1, 256, 0, st>>>(ctl, act, nmember);
  count_launches(1);
}

}  // namespace xm
