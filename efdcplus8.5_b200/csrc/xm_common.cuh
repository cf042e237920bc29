// xm_common.cuh -- device helpers shared by the kernel files.
#pragma once

#include "xm_internal.h"

namespace xm {

// Slot of a cell and of its four neighbours (tile layout, see xm_internal.h).
struct Nb {
  int d, e, w, n, s;
};

__device__ __forceinline__ Nb neighbours(const int4 *__restrict__ tnbr, int tile, int tid) {
  const int tx = tid & (TX - 1), ty = tid >> 5;
  const int4 nb = __ldg(&tnbr[tile]);  // (w, e, s, n)
  Nb r;
  r.d = tile * TILE + tid;
  r.e = (tx < TX - 1) ? r.d + 1 : nb.y * TILE + ty * TX;
  r.w = (tx > 0) ? r.d - 1 : nb.x * TILE + ty * TX + (TX - 1);
  r.n = (ty < TY - 1) ? r.d + TX : nb.w * TILE + tx;
  r.s = (ty > 0) ? r.d - TX : nb.z * TILE + (TY - 1) * TX + tx;
  return r;
}

__device__ __forceinline__ Nb neighbours_of_slot(const int4 *__restrict__ tnbr, int d) {
  return neighbours(tnbr, d / TILE, d % TILE);
}

// Block-wide sum of NT threads, fixed tree order; result valid in thread 0.
template <class T>
__device__ __forceinline__ T block_sum(T v, T *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < NT / 32) ? sh[lane] : T(0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

__device__ __forceinline__ double block_min(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = (lane < NT / 32) ? sh[lane] : 1.e+18;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  }
  return v;
}

// "Last CTA" arrival: every CTA publishes its partials, then the CTA that
// arrives last returns true (in all its threads) and may reduce them.
__device__ __forceinline__ bool arrive_last(unsigned int *counter) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int prev = atomicAdd(counter, 1u);
    last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Fixed-order sum of nblk partials by the last CTA: thread i adds partials
// i, i+NT, ... in order, then the fixed block tree.  Deterministic.
__device__ __forceinline__ double reduce_partials(const double *part, int nblk, double *sh) {
  double s = 0.0;
  for (int i = threadIdx.x; i < nblk; i += NT) s += __ldcg(&part[i]);
  return block_sum(s, sh);
}

}  // namespace xm
