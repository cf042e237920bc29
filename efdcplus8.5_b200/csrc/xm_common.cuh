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

// Fixed-order sum of nblk partials by one CTA: thread i adds partials
// i, i+NT, ... in order, then the fixed block tree.  Deterministic; W, the
// loads a thread issues before adding them (in order), changes only speed
// and registers.
template <int W = 8>
__device__ __forceinline__ double reduce_partials(const double *part, int nblk, double *sh) {
  double s = 0.0;
  for (int base = 0; base < nblk; base += W * NT) {
    double v[W];  // a pass's loads are all issued before the (ordered) adds
#pragma unroll
    for (int j = 0; j < W; ++j) {
      const int i = base + j * NT + int(threadIdx.x);
      v[j] = (i < nblk) ? __ldcg(&part[i]) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < W; ++j) s += v[j];
  }
  return block_sum(s, sh);
}

// atomic min of a non-negative double (its bit pattern orders like its value)
__device__ __forceinline__ void atomic_min_nonneg(double *addr, double v) {
  atomicMin(reinterpret_cast<unsigned long long *>(addr),
            static_cast<unsigned long long>(__double_as_longlong(fmax(v, 0.0))));
}

// ---------------------------------------------------------------------------
// Row-vector geometry of the CG kernels: a thread owns 4 consecutive cells of
// one tile row (8 threads per row, 64 per tile, 4 tiles per 256-thread CTA).
// Row vectors are 16 B (FP32) / 32 B (FP64) aligned, so they move as 128-bit
// loads; the E/W neighbours of the vector come from the adjacent lanes of the
// row (warp shuffles) and, at the tile edge, from the neighbour tile.
constexpr int CPT = 4;              // cells per thread
constexpr int ROWT = TX / CPT;      // threads per row (8)
constexpr int TPT = TILE / CPT;     // threads per tile (64)
constexpr int TILES_PER_CTA = NT / TPT;  // 4

struct RowGeo {
  int d0;      // first slot of the thread's 4 cells
  int dn, ds;  // first slots of the same 4 columns in the rows above / below
  int dwe;     // slot west of cell 0 (used when cx == 0)
  int dee;     // slot east of cell 3 (used when cx == ROWT-1)
  int cx;      // column group 0..7
};

// nb = tnbr[tile], the (w, e, s, n) neighbour tiles
__device__ __forceinline__ RowGeo row_geo_nb(const int4 nb, int tile, int q) {
  const int cx = q & (ROWT - 1), ty = q / ROWT;
  RowGeo g;
  g.cx = cx;
  g.d0 = tile * TILE + ty * TX + cx * CPT;
  g.dn = (ty < TY - 1) ? g.d0 + TX : nb.w * TILE + cx * CPT;
  g.ds = (ty > 0) ? g.d0 - TX : nb.z * TILE + (TY - 1) * TX + cx * CPT;
  g.dwe = nb.x * TILE + ty * TX + (TX - 1);
  g.dee = nb.y * TILE + ty * TX;
  return g;
}

__device__ __forceinline__ RowGeo row_geo(const int4 *__restrict__ tnbr, int tile, int q) {
  return row_geo_nb(__ldg(&tnbr[tile]), tile, q);
}

template <class T>
struct V4 {
  T x, y, z, w;
};

__device__ __forceinline__ V4<float> ld4(const float *p) {
  const float4 v = *reinterpret_cast<const float4 *>(p);
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ V4<double> ld4(const double *p) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0];
  const double2 b = reinterpret_cast<const double2 *>(p)[1];
  return {a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ void st4(float *p, const V4<float> &v) {
  *reinterpret_cast<float4 *>(p) = make_float4(v.x, v.y, v.z, v.w);
}
__device__ __forceinline__ void st4(double *p, const V4<double> &v) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(v.x, v.y);
  reinterpret_cast<double2 *>(p)[1] = make_double2(v.z, v.w);
}

// value of the west neighbour of cell 0 / east neighbour of cell 3, from the
// adjacent lane of the row (the tile-edge lanes substitute their own load)
template <class T>
__device__ __forceinline__ T from_west(const V4<T> &v) {
  return __shfl_up_sync(0xffffffffu, v.w, 1, ROWT);
}
template <class T>
__device__ __forceinline__ T from_east(const V4<T> &v) {
  return __shfl_down_sync(0xffffffffu, v.x, 1, ROWT);
}

}  // namespace xm
