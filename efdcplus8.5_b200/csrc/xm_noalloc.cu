// xm_noalloc.cu -- CONGRAD that allocates nothing (efdc_xm_congrad_noalloc).
//
// Who needs it: callers that cannot let a library allocate device memory --
// a host code that hands all of its GPU memory to its own pool or budget, a
// caller inside a time-critical loop where an allocation could stall or fail,
// or one that only has device arrays it manages itself (CUDA Fortran device
// arrays, a framework's tensors).  They pass device arrays for the system and
// the solution; the solver's own vectors live in one fixed-size array of
// device memory declared at file scope below, which exists on every GPU that
// loads this library, from the library's loading until the process exits.
//
// Everything else in the library (efdc_xm_create and the context API) is
// unchanged; this file adds one entry point beside them.
//
// The algorithm is CONGRAD's Jacobi-preconditioned CG (congrad.f90:54-187) in
// FP64 on the reference's own layout: cells L=2..LA in CELLMAP order with the
// LNC/LSC/LEC/LWC neighbour maps (so periodic links work too), one thread per
// cell, three kernels per iteration like the reference's three loops.

#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/efdc_xm.h"
#include "xm_common.cuh"
#include "xm_kernels.h"

namespace {

constexpr int NA_MAX_CELLS = EFDC_XM_NOALLOC_MAX_CELLS;  // water cells, LA-1
constexpr int NA_LEN = ((NA_MAX_CELLS + 2 + 31) / 32) * 32;  // elements 1..LC, padded
constexpr int NA_GRID = 296;                          // CTAs (2 per SM of a B200)
constexpr int NA_CTL = 16;                            // doubles of the control block
constexpr size_t NA_DOUBLES = size_t(3) * NA_LEN + 2 * NA_GRID + NA_CTL;

// The scratch: r | p | Ap | partial sums | control block.  In host code this
// name is only a stand-in for the symbol; its device address comes from
// cudaGetSymbolAddress (see scratch_ptr).
static __device__ __align__(256) double g_na_scratch[NA_DOUBLES];

struct NaCtl {  // lives in the last NA_CTL doubles of the scratch
  double rpcg, alpha, beta, rsq;
  int iter, done, status, pad;
  unsigned int counter, pad2;
};
static_assert(sizeof(NaCtl) <= NA_CTL * sizeof(double), "control block too large");

struct NaArgs {
  int la, lc;
  const int *lnc, *lsc, *lec, *lwc;
  const double *ccc, *ccs, *ccn, *ccw, *cce, *fptmp;
  double *P;
  double *r, *p, *ap, *part;
  NaCtl *ctl;
};

using xm::arrive_last;
using xm::block_sum;
using xm::NT;
using xm::reduce_partials;

// :54-88 RCG = FPTMP - A*P; PCG = RCG*CCCI; RPCG.  Also zeroes the ghost
// elements 1 and LC of PCG (congrad.f90:42: PCG(1)=PCG(LC)=0).
__global__ void __launch_bounds__(NT) k_na_init(NaArgs a) {
  __shared__ double sh[32];
  double acc = 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.p[0] = 0.0;
    a.p[a.lc - 1] = 0.0;
  }
  for (int L = 2 + blockIdx.x * NT + threadIdx.x; L <= a.la; L += gridDim.x * NT) {
    const int i = L - 1;
    const double r = a.fptmp[i] - a.ccc[i] * a.P[i] - a.ccn[i] * a.P[a.lnc[i] - 1] -
                     a.ccs[i] * a.P[a.lsc[i] - 1] - a.ccw[i] * a.P[a.lwc[i] - 1] -
                     a.cce[i] * a.P[a.lec[i] - 1];
    const double z = r * (1. / a.ccc[i]);
    a.r[i] = r;
    a.p[i] = z;
    acc += r * z;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) a.part[blockIdx.x] = acc;
  if (arrive_last(&a.ctl->counter)) {
    const double rpcg = reduce_partials<>(a.part, gridDim.x, sh);
    if (threadIdx.x == 0) {
      a.ctl->rpcg = rpcg;
      a.ctl->iter = 0;
      a.ctl->status = 0;
      a.ctl->done = (rpcg == 0.0) ? 1 : 0;
      if (!isfinite(rpcg)) {
        a.ctl->done = 1;
        a.ctl->status = EFDC_XM_NONFINITE;
      }
      a.ctl->counter = 0;
    }
  }
}

// :107-125 APCG and ALPHA
__global__ void __launch_bounds__(NT) k_na_matvec(NaArgs a) {
  __shared__ double sh[32];
  if (a.ctl->done) return;
  double acc = 0.0;
  for (int L = 2 + blockIdx.x * NT + threadIdx.x; L <= a.la; L += gridDim.x * NT) {
    const int i = L - 1;
    const double p = a.p[i];
    const double ap = a.ccc[i] * p + a.ccs[i] * a.p[a.lsc[i] - 1] + a.ccn[i] * a.p[a.lnc[i] - 1] +
                      a.ccw[i] * a.p[a.lwc[i] - 1] + a.cce[i] * a.p[a.lec[i] - 1];
    a.ap[i] = ap;
    acc += ap * p;
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) a.part[blockIdx.x] = acc;
  if (arrive_last(&a.ctl->counter)) {
    const double papcg = reduce_partials<>(a.part, gridDim.x, sh);
    if (threadIdx.x == 0) {
      a.ctl->alpha = a.ctl->rpcg / papcg;
      a.ctl->counter = 0;
    }
  }
}

// :127-149 P, RCG, RPCGN, RSQ, BETA and the stop test
__global__ void __launch_bounds__(NT) k_na_update(NaArgs a, double rsqm, int iterm) {
  __shared__ double sh[32];
  if (a.ctl->done) return;
  const double alpha = a.ctl->alpha;
  double a1 = 0.0, a2 = 0.0;
  for (int L = 2 + blockIdx.x * NT + threadIdx.x; L <= a.la; L += gridDim.x * NT) {
    const int i = L - 1;
    a.P[i] = a.P[i] + alpha * a.p[i];
    const double r = a.r[i] - alpha * a.ap[i];
    a.r[i] = r;
    const double z = (1. / a.ccc[i]) * r;
    a1 += r * z;
    a2 += r * r;
  }
  a1 = block_sum(a1, sh);
  if (threadIdx.x == 0) a.part[blockIdx.x] = a1;
  a2 = block_sum(a2, sh);
  if (threadIdx.x == 0) a.part[gridDim.x + blockIdx.x] = a2;
  if (arrive_last(&a.ctl->counter)) {
    const double rpcgn = reduce_partials<>(a.part, gridDim.x, sh);
    const double rsq = reduce_partials<>(a.part + gridDim.x, gridDim.x, sh);
    if (threadIdx.x == 0) {
      a.ctl->beta = rpcgn / a.ctl->rpcg;
      a.ctl->rpcg = rpcgn;
      a.ctl->rsq = rsq;
      const int it = a.ctl->iter + 1;
      a.ctl->iter = it;
      if (!isfinite(rsq) || !isfinite(a.ctl->alpha)) {
        a.ctl->done = 1;
        a.ctl->status = EFDC_XM_NONFINITE;
      } else if (rsq <= rsqm) {
        a.ctl->done = 1;
      } else if (it >= iterm) {
        a.ctl->done = 1;
        a.ctl->status = EFDC_XM_CG_MAXITER;
      }
      a.ctl->counter = 0;
    }
  }
}

// :151-162 PCG = TMPCG + BETA*PCG
__global__ void __launch_bounds__(NT) k_na_pupdate(NaArgs a) {
  if (a.ctl->done) return;
  const double beta = a.ctl->beta;
  for (int L = 2 + blockIdx.x * NT + threadIdx.x; L <= a.la; L += gridDim.x * NT) {
    const int i = L - 1;
    a.p[i] = (1. / a.ccc[i]) * a.r[i] + beta * a.p[i];
  }
}

thread_local char g_na_msg[512];

// the message goes to efdc_xm_last_error(), shared with the rest of the ABI
void na_error(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
void na_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_na_msg, sizeof(g_na_msg), fmt, ap);
  va_end(ap);
  xm::set_last_error_str(g_na_msg);
}

// Device address of the scratch, looked up once per device (with that
// device current) and kept for the life of the process.
std::mutex g_na_mutex;
double *g_na_ptr[64] = {nullptr};

int scratch_ptr(int dev, double **out) {
  if (dev < 0 || dev >= 64) {
    na_error("efdc_xm_congrad_noalloc: device %d out of range", dev);
    return EFDC_XM_BAD_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess || !p) {
      na_error("efdc_xm_congrad_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
               cudaGetErrorString(e));
      return EFDC_XM_CUDA_ERROR;
    }
    g_na_ptr[dev] = static_cast<double *>(p);
  }
  *out = g_na_ptr[dev];
  return EFDC_XM_OK;
}

}  // namespace

extern "C" {

int32_t efdc_xm_congrad_noalloc(int32_t la, const int32_t *lnc, const int32_t *lsc,
                                const int32_t *lec, const int32_t *lwc, const double *ccc,
                                const double *ccs, const double *ccn, const double *ccw,
                                const double *cce, const double *fptmp, double *p, double rsqm,
                                int32_t iterm, void *stream, int32_t *iters, double *rsq) {
  if (la < 2 || iterm < 1 || !lnc || !lsc || !lec || !lwc || !ccc || !ccs || !ccn || !ccw ||
      !cce || !fptmp || !p) {
    na_error("efdc_xm_congrad_noalloc: need LA >= 2, ITERM >= 1 and non-NULL device arrays");
    return EFDC_XM_BAD_ARGUMENT;
  }
  if (la - 1 > NA_MAX_CELLS) {
    na_error("efdc_xm_congrad_noalloc: LA-1 = %d water cells exceeds the fixed scratch of %d "
             "cells; use efdc_xm_create/efdc_xm_congrad for larger systems", la - 1, NA_MAX_CELLS);
    return EFDC_XM_BAD_ARGUMENT;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  double *base = nullptr;
  int rc = (e == cudaSuccess) ? scratch_ptr(dev, &base) : EFDC_XM_CUDA_ERROR;
  if (rc) {
    if (e != cudaSuccess)
      na_error("efdc_xm_congrad_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    return rc;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  NaArgs a;
  a.la = la;
  a.lc = la + 1;
  a.lnc = lnc;
  a.lsc = lsc;
  a.lec = lec;
  a.lwc = lwc;
  a.ccc = ccc;
  a.ccs = ccs;
  a.ccn = ccn;
  a.ccw = ccw;
  a.cce = cce;
  a.fptmp = fptmp;
  a.P = p;
  a.r = base;
  a.p = base + NA_LEN;
  a.ap = base + 2 * size_t(NA_LEN);
  a.part = base + 3 * size_t(NA_LEN);
  a.ctl = reinterpret_cast<NaCtl *>(base + 3 * size_t(NA_LEN) + 2 * NA_GRID);
  const int grid = std::max(1, std::min(NA_GRID, (la - 1 + NT - 1) / NT));
  // the control block keeps the previous call's contents: start from zero
  auto fail = [&](cudaError_t err, const char *what) {
    na_error("efdc_xm_congrad_noalloc: %s: %s", what, cudaGetErrorString(err));
    return EFDC_XM_CUDA_ERROR;
  };
  if ((e = cudaMemsetAsync(a.ctl, 0, sizeof(NaCtl), st)) != cudaSuccess) return fail(e, "memset");
  k_na_init<<<grid, NT, 0, st>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "launch");
  NaCtl h{};
  int launched = 0;
  while (launched < iterm) {
    const int chunk = std::min(8, iterm - launched);
    for (int k = 0; k < chunk; ++k) {
      k_na_matvec<<<grid, NT, 0, st>>>(a);
      k_na_update<<<grid, NT, 0, st>>>(a, rsqm, iterm);
      k_na_pupdate<<<grid, NT, 0, st>>>(a);
    }
    launched += chunk;
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "launch");
    if ((e = cudaMemcpyAsync(&h, a.ctl, sizeof(NaCtl), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return fail(e, "copy of the control block");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(e, "synchronize");
    if (h.done) break;
  }
  if (iters) *iters = h.iter;
  if (rsq) *rsq = h.rsq;
  if (!h.done) return EFDC_XM_CG_MAXITER;
  if (h.status == EFDC_XM_CG_MAXITER)
    na_error("efdc_xm_congrad_noalloc: maximum iterations exceeded (RSQ=%g)", h.rsq);
  if (h.status == EFDC_XM_NONFINITE)
    na_error("efdc_xm_congrad_noalloc: non-finite CG scalars at iteration %d", h.iter);
  return h.status;
}

}  // extern "C"
