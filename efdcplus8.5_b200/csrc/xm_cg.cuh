// xm_cg.cuh -- bodies of the CG iteration kernels, shared by the FP64 drop-in
// (xm_step.cu, compiled without FMA contraction so each statement rounds as in
// congrad.f90) and the FP32 inner solve of the MIXED form (xm_mixed.cu).
//
// A thread owns 4 consecutive cells of a tile row (see RowGeo).  Land slots
// are inert by construction (r = p = 0, CCC = 1, couplings 0), so the cell
// loops run unconditionally; only the residual kernels, which read P at
// land slots (P(LC), the ghost value), mask with the slot kind.
#pragma once

#include <type_traits>

#include "../../include/efdc_xm.h"
#include "xm_common.cuh"
#include "xm_tma.cuh"

namespace xm {

__device__ __forceinline__ float rcpT(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcpT(double x) { return 1. / x; }

// The CG kernels loop over "quads": 4 consecutive tiles of one member, one
// CTA pass each (a thread owns 4 cells of a row, 64 threads per tile), quads
// dealt to the CTAs cyclically.  Past the member's last tile a thread works
// on tile 0 (member 0's ghost tile, all inert) with stores off, so that every lane
// of a row takes part in the shuffles.  A quad whose member is finished (or
// not in this sweep) is skipped by the whole CTA.
//
// Reductions: the CG kernel leaves one partial per warp in shared memory
// (warp shuffles only, no CTA barrier per quad) and, every QCAP quads and at
// its end, adds the warp partials of each quad in fixed warp order into
// part[quad] (plain stores).  Each member's per-quad partials are then summed
// in fixed quad order and the member finished (its Ctl), either
//  * folded into the CG kernel (Fold): each stored quad counts towards its
//    member's arrivals (Ctl::counter, after a fence), and the CTA whose store
//    completes a member's quads sums that member and runs its epilogue, or
//  * by a member-reduce kernel after it (one CTA per member), where sub-grid
//    channel kernels add their terms to the partials in between.
// Both run the same sum (reduce_partials) and the same epilogue, so the two
// forms give the same iterates bit for bit, and neither depends on the grid
// size or on which other members share the context.
// A member's operator is handled as unsymmetric (the four-array form) when
// its flag's bit 1 is set; MA = false compiles the symmetric form only, for
// batches in which no member can be unsymmetric (no radiation boundary).
template <bool MA>
__device__ __forceinline__ bool unsym(const Ctl &k) {
  return MA && (k.asym & 1) != 0;
}

constexpr int QCAP = 32;         // quads a CTA logs between two stores
constexpr int NWARP = NT / 32;   // warps per CTA

template <int NS>
struct QuadLog {
  double w[NS][QCAP][NWARP];  // per-warp partials of NS sums
  int qd[QCAP];               // quad of each entry
  int m[QCAP];                // its member
};

// atomicAdd with acquire-release semantics at GPU scope: the partial sums
// this thread stored are visible to whoever observes the increment, and
// those the earlier arrivals stored are visible to this thread.
__device__ __forceinline__ unsigned int atomic_add_acq_rel(unsigned int *p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
               : "=r"(old)
               : "l"(p), "r"(v)
               : "memory");
  return old;
}

// The member reduction folded into a CG kernel: ctl holds the members'
// arrival counters and epi(m, sums) finishes member m (all threads call it;
// the sums are valid in thread 0).  Fold<NoEpi>: not folded, a member-reduce
// kernel follows.
template <class Epi>
struct Fold {
  Ctl *ctl;
  Epi epi;
};
struct NoEpi {
  __device__ void operator()(int, const double *) const {}
};
// What the epilogues of the update and residual kernels read besides the Ctl
// (kernel arguments of the folded form and of the member-reduce kernels).
struct RedArgs {
  Glob *glob;
  double rsqm_fac, rel_tol, margin;  // MIXED refinement residual (k_mx_resid)
  int no_stop;                       // iterate past the stop tests (kernel timing)
  int unscaled;                      // MIXED residual of the unscaled system
};
__device__ __forceinline__ Fold<NoEpi> no_fold() { return Fold<NoEpi>{nullptr, NoEpi{}}; }
// The fold of a kernel compiled with FOLD, else none (the kernel then has no
// trace of it: no counters, no atomics, no registers held for it).
template <bool FOLD, class Epi>
__device__ __forceinline__ auto fold_if(Ctl *ctl, Epi epi) {
  if constexpr (FOLD)
    return Fold<Epi>{ctl, epi};
  else
    return no_fold();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int NS, class Epi>
__device__ __forceinline__ void quad_store(QuadLog<NS> &L, int n, const DevStatic &S,
                                           double *part, const Fold<Epi> &f) {
  constexpr bool kFold = !std::is_same<Epi, NoEpi>::value;
  __shared__ int nfin;
  __shared__ int fin[QCAP];
  __shared__ double sh[32];
  if constexpr (kFold) {
    if (threadIdx.x == 0) nfin = 0;
  }
  __syncthreads();  // the warp partials and the entries are in shared memory
  const int t = threadIdx.x;
  if (t < n) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      double a = 0.0;
#pragma unroll
      for (int w = 0; w < NWARP; ++w) a += L.w[s][t][w];
      part[size_t(s) * S.nquad + L.qd[t]] = a;
    }
    if constexpr (kFold) {  // this quad arrives (release: after its partials)
      const int m = L.m[t];
      const unsigned int nq = unsigned(S.qstart[m + 1] - S.qstart[m]);
      if (atomic_add_acq_rel(&f.ctl[m].counter, 1u) == nq - 1u) fin[atomicAdd(&nfin, 1)] = m;
    }
  }
  __syncthreads();  // the log is reused after this (folded: the list is complete, and the
                    // acquiring threads' view orders the CTA's reads below)
  if constexpr (kFold) {
    const int k = nfin;
    for (int i = 0; i < k; ++i) {  // the members this CTA completed (any order)
      const int m = fin[i];
      const int q0 = S.qstart[m], nq = S.qstart[m + 1] - q0;
      double r[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s)
        r[s] = reduce_partials<>(part + size_t(s) * S.nquad + q0, nq, sh);
      f.epi(m, r);
      if (t == 0) f.ctl[m].counter = 0u;  // for the next kernel
    }
    __syncthreads();  // the list is reused after this
  }
}

// One CG kernel over all quads.  setup(m) returns the member's values for the
// body (a struct with at least `bool skip`).  body(a, g, valid, v) processes
// one quad row vector and adds its parts of the NS sums to v[].
//
// Everything a quad's loads depend on (its table entry, its member's values
// from setup() and the thread's tile-neighbour entry)
// is fetched one quad ahead, so that those small dependent loads overlap the
// current quad's memory traffic instead of preceding the next one's.  In an
// ensemble nearly every quad of a CTA belongs to another member.
template <int NS, class Setup, class Body, class Epi = NoEpi>
__device__ __forceinline__ void quad_sweep(const DevStatic &S, double *part, Setup setup,
                                           Body body, Fold<Epi> f = no_fold()) {
  __shared__ QuadLog<NS> L;
  const int sub = threadIdx.x / TPT, q = threadIdx.x % TPT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int G = gridDim.x, NQ = S.nquad;
  int qd = blockIdx.x;
  if (qd >= NQ) return;
  int4 cur = S.quads[qd];
  auto a = setup(cur.x);
  int4 nb = __ldg(&S.tnbr[sub < cur.z ? cur.y + sub : 0]);
  int4 nxt = (qd + G < NQ) ? S.quads[qd + G] : cur;
  int n = 0;
  for (;;) {
    const int qn = qd + G;
    const bool more = qn < NQ;
    // the next quad's descriptors (one load level after its table entry)
    auto an = a;
    if (more && nxt.x != cur.x) an = setup(nxt.x);
    const int4 nbn = __ldg(&S.tnbr[(more && sub < nxt.z) ? nxt.y + sub : 0]);
    const int4 nn = (qn + G < NQ) ? S.quads[qn + G] : nxt;
    if (!a.skip) {
      const int ti = cur.y + sub;
      const bool valid = sub < cur.z;
      const RowGeo g = row_geo_nb(nb, valid ? ti : 0, q);
      double v[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) v[s] = 0.0;
      body(a, g, valid, v);
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double x = warp_sum(v[s]);
        if (lane == 0) L.w[s][n][warp] = x;
      }
      if (threadIdx.x == 0) {
        L.qd[n] = qd;
        if constexpr (!std::is_same<Epi, NoEpi>::value) L.m[n] = cur.x;
      }
      if (++n == QCAP) {
        quad_store<NS>(L, n, S, part, f);
        n = 0;
      }
    }
    if (!more) break;
    qd = qn;
    cur = nxt;
    a = an;
    nb = nbn;
    nxt = nn;
  }
  if (n) quad_store<NS>(L, n, S, part, f);
}

// quad_sweep with the descriptors in batches: the CTA first loads, for its
// next QB quads at once, each quad's table entry, its member's values and its
// tiles' neighbour entries into shared memory (one round of dependent loads
// per batch, by QB*4 threads in parallel), then runs the quads with no
// dependent load ahead of their data loads.  Same results as quad_sweep: the
// same rows, the same warp sums, the same per-quad partials.
constexpr int QB = 32;  // quads per descriptor batch (QB * TILES_PER_CTA <= NT)

template <int NS, class Setup, class Body, class Epi>
__device__ __forceinline__ void quad_sweep_batched(const DevStatic &S, double *part, Setup setup,
                                                   Body body, const Fold<Epi> &f) {
  using A = decltype(setup(0));
  __shared__ QuadLog<NS> L;
  __shared__ A da[QB];
  __shared__ int4 dq[QB];
  __shared__ int4 dnb[QB][TILES_PER_CTA];
  static_assert(QB * TILES_PER_CTA <= NT, "one descriptor load per thread");
  const int sub = threadIdx.x / TPT, q = threadIdx.x % TPT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int G = gridDim.x, NQ = S.nquad;
  int n = 0;
  for (int b0 = blockIdx.x; b0 < NQ; b0 += G * QB) {
    __syncthreads();  // the previous batch's descriptors are no longer read
    if (threadIdx.x < QB * TILES_PER_CTA) {
      const int k = threadIdx.x / TILES_PER_CTA, s = threadIdx.x % TILES_PER_CTA;
      const int qd = b0 + k * G;
      if (qd < NQ) {
        const int4 cur = S.quads[qd];
        if (s == 0) {
          dq[k] = cur;
          da[k] = setup(cur.x);
        }
        dnb[k][s] = __ldg(&S.tnbr[s < cur.z ? cur.y + s : 0]);
      }
    }
    __syncthreads();
    const int nk = min(QB, (NQ - b0 + G - 1) / G);
    for (int k = 0; k < nk; ++k) {
      const A a = da[k];
      if (a.skip) continue;  // the same for the whole CTA
      const int4 cur = dq[k];
      const bool valid = sub < cur.z;
      const RowGeo g = row_geo_nb(dnb[k][sub], valid ? cur.y + sub : 0, q);
      double v[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) v[s] = 0.0;
      body(a, g, valid, v);
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double x = warp_sum(v[s]);
        if (lane == 0) L.w[s][n][warp] = x;
      }
      if (threadIdx.x == 0) {
        L.qd[n] = b0 + k * G;
        if constexpr (!std::is_same<Epi, NoEpi>::value) L.m[n] = cur.x;
      }
      if (++n == QCAP) {
        quad_store<NS>(L, n, S, part, f);
        n = 0;
      }
    }
  }
  if (n) quad_store<NS>(L, n, S, part, f);
}

// ---------------------------------------------------------------------------
// Staged quad sweep (FP32 kernels, variant 2).  A quad's tiles of NB arrays
// (1 KB per tile and array, contiguous because a quad's tiles are) move into
// shared memory by 1-D bulk copies that complete on an mbarrier, in a ring of
// NSTG stages: while the CTA computes one quad, the copies of the next
// NSTG - 1 quads are in flight.  The rows outside the quad's tiles -- the N/S
// halo rows of a tile's edge rows and the E/W edge columns -- are plain loads
// issued before the wait (L2 hits: the neighbour tiles are in flight or just
// done in the same window of quads).  Only this GPU's memory is read, each
// CTA for itself: no multicast.
template <int NB>
struct Stage {
  float body[NB][TILES_PER_CTA * TILE];
};

// Where a thread's cells are in a stage, and whether its N/S rows are outside
// the tile (row 7: the N row is the north tile's row 0; row 0: the S row is
// the south tile's row 7).
struct StageRow {
  int r0;
  bool north, south;
};

__device__ __forceinline__ StageRow stage_row(int sub, int q) {
  const int cx = q & (ROWT - 1), ty = q / ROWT;
  return StageRow{sub * TILE + ty * TX + cx * CPT, ty == TY - 1, ty == 0};
}

template <int NB>
__device__ __forceinline__ V4<float> st_body(const Stage<NB> &st, int i, const StageRow &r) {
  return ld4(&st.body[i][r.r0]);
}
// the row above the thread's cells in array i: in the stage, or `halo`
template <int NB>
__device__ __forceinline__ V4<float> st_north(const Stage<NB> &st, int i, const StageRow &r,
                                              const V4<float> &halo) {
  return r.north ? halo : ld4(&st.body[i][r.r0 + TX]);
}
template <int NB>
__device__ __forceinline__ V4<float> st_south(const Stage<NB> &st, int i, const StageRow &r,
                                              const V4<float> &halo) {
  return r.south ? halo : ld4(&st.body[i][r.r0 - TX]);
}

constexpr int MBAR_TRIES = 1 << 16;  // bounded mbarrier waits (each try may suspend)

// setup(m) returns the member's values (a struct with `bool skip` and the NB
// source arrays `const float *b[NB]`); pre(a, g, row) loads the thread's
// halo rows and edge values from global memory before the stage is waited
// for; body(a, st, row, g, valid, e, v) computes one quad row vector from
// stage st and those values e.  On a wait that runs out, *err is set and the
// CTA stops computing (the step then fails with a timeout status); the copies
// it issued are waited for, again bounded, before it exits.
template <int NS, int NB, int NSTG, class Setup, class Pre, class Body, class Epi>
__device__ __forceinline__ void quad_sweep_staged(const DevStatic &S, double *part, int *err,
                                                  Setup setup, Pre pre, Body body,
                                                  const Fold<Epi> &f) {
  using A = decltype(setup(0));
  using St = Stage<NB>;
  extern __shared__ __align__(128) unsigned char dyn_smem[];
  St *stg = reinterpret_cast<St *>(dyn_smem);
  __shared__ __align__(8) uint64_t bar[NSTG];
  __shared__ QuadLog<NS> L;
  __shared__ A da[QB];
  __shared__ int4 dq[QB];
  __shared__ int4 dnb[QB][TILES_PER_CTA];
  __shared__ int list[QB];
  __shared__ int nlist;
  const int sub = threadIdx.x / TPT, q = threadIdx.x % TPT;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int G = gridDim.x, NQ = S.nquad;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NSTG; ++i) mbar_init(&bar[i], 1);
    mbar_fence_init();
  }
  __syncthreads();
  uint32_t phase = 0;  // bit i: parity of stage i's next phase
  bool dead = false;   // a wait ran out
  const StageRow row = stage_row(sub, q);
  // thread 0: the copies of list entry j into stage j % NSTG
  auto issue = [&](int j) {
    const int k = list[j], s = j % NSTG;
    const int4 cur = dq[k];
    const A &a = da[k];
    const uint32_t bb = uint32_t(cur.z) * TILE * sizeof(float);
    mbar_arrive_expect(&bar[s], NB * bb);
    const size_t off = size_t(cur.y) * TILE;
#pragma unroll
    for (int i = 0; i < NB; ++i) bulk_g2s(stg[s].body[i], a.b[i] + off, bb, &bar[s]);
  };
  int n = 0;
  for (int b0 = blockIdx.x; b0 < NQ; b0 += G * QB) {
    __syncthreads();  // the previous batch's descriptors are no longer read
    if (threadIdx.x < QB * TILES_PER_CTA) {
      const int k = threadIdx.x / TILES_PER_CTA, s = threadIdx.x % TILES_PER_CTA;
      const int qd = b0 + k * G;
      if (qd < NQ) {
        const int4 cur = S.quads[qd];
        if (s == 0) {
          dq[k] = cur;
          da[k] = setup(cur.x);
        }
        dnb[k][s] = __ldg(&S.tnbr[s < cur.z ? cur.y + s : 0]);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // the quads of the batch that run, in order
      const int nk = min(QB, (NQ - b0 + G - 1) / G);
      int c = 0;
      for (int k = 0; k < nk; ++k)
        if (!da[k].skip) list[c++] = k;
      nlist = c;
      if (!dead)
        for (int j = 0; j < NSTG && j < c; ++j) issue(j);
    }
    __syncthreads();
    const int nl = nlist;
    for (int j = 0; j < nl; ++j) {
      const int k = list[j], s = j % NSTG;
      const A a = da[k];
      const int4 cur = dq[k];
      const bool valid = sub < cur.z;
      const RowGeo g = row_geo_nb(dnb[k][sub], valid ? cur.y + sub : 0, q);
      const auto e = pre(a, g, row);
      if (!dead && !mbar_wait(&bar[s], (phase >> s) & 1u, MBAR_TRIES)) dead = true;
      phase ^= 1u << s;
      double v[NS];
#pragma unroll
      for (int i = 0; i < NS; ++i) v[i] = 0.0;
      if (!dead) body(a, stg[s], row, g, valid, e, v);
#pragma unroll
      for (int i = 0; i < NS; ++i) {
        const double x = warp_sum(v[i]);
        if (lane == 0) L.w[i][n][warp] = x;
      }
      if (threadIdx.x == 0) {
        L.qd[n] = b0 + k * G;
        if constexpr (!std::is_same<Epi, NoEpi>::value) L.m[n] = cur.x;
      }
      __syncthreads();  // every thread is done with stage s: it may be refilled
      if (threadIdx.x == 0 && !dead && j + NSTG < nl) issue(j + NSTG);
      if (++n == QCAP) {
        quad_store<NS>(L, n, S, part, f);
        n = 0;
      }
    }
  }
  if (n) quad_store<NS>(L, n, S, part, f);
  // every phase issued has been waited for, unless a wait ran out: then the
  // copies still in flight are waited for (bounded) before the CTA's shared
  // memory goes
  if (dead && threadIdx.x == 0) {
    atomicExch(err, 1);
#pragma unroll
    for (int i = 0; i < NSTG; ++i) mbar_wait(&bar[i], (phase >> i) & 1u, MBAR_TRIES);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NSTG; ++i) mbar_inval(&bar[i]);
  }
}

// The quad sweep of a kernel variant: 0 prefetches one quad ahead in
// registers, 1 and 3 load the descriptors in batches (quad_sweep_batched).
template <int NS, int VAR, class Setup, class Body, class Epi>
__device__ __forceinline__ void quad_sweep_v(const DevStatic &S, double *part, Setup setup,
                                             Body body, const Fold<Epi> &f) {
  if constexpr (VAR == 1 || VAR == 3)
    quad_sweep_batched<NS>(S, part, setup, body, f);
  else
    quad_sweep<NS>(S, part, setup, body, f);
}

// The members' epilogues of the reductions (thread 0 of the member), run by
// the member-reduce kernels and by the folded form alike.
// FP64 CONGRAD (congrad.f90): :88 RETURN on RPCG = 0; :124 ALPHA (also the
// MIXED inner ALPHA); :143-169 BETA, RSQ and the stop test.  With no_stop the
// iteration continues past RSQM and ITERM (kernel timing).
__device__ __forceinline__ void cg_init_epi(Ctl &k, Glob *glob, double rpcg) {
  k.rpcg = rpcg;
  k.beta = 0.0;
  k.parity = 0;
  k.iter = 0;
  k.rsq = 0.0;
  k.status = 0;
  if (rpcg == 0.0 || !isfinite(rpcg)) {  // :88 RETURN
    if (!isfinite(rpcg)) k.status = EFDC_XM_NONFINITE;
    k.done = 1;
    atomicAdd(&glob->ndone, 1);
  }
}
__device__ __forceinline__ void cg_matvec_epi(Ctl &k, double pap) {
  k.papcg = pap;
  k.alpha = k.rpcg / pap;  // :124
}
__device__ __forceinline__ void cg_update_epi(Ctl &k, Glob *glob, const StepScalars &c,
                                              double rpcgn, double rsq, int no_stop) {
  k.beta = rpcgn / k.rpcg;
  k.rpcg = rpcgn;
  k.rsq = rsq;
  const int it = k.iter + 1;
  k.iter = it;
  int fin = 0;
  if (!isfinite(rsq) || !isfinite(k.alpha)) {
    k.status = EFDC_XM_NONFINITE;
    fin = 1;
  } else if (!no_stop && rsq <= c.rsqm) {
    fin = 1;
  } else if (!no_stop && it >= c.iterm) {
    k.status = EFDC_XM_CG_MAXITER;
    fin = 1;
  } else {
    k.parity ^= 1;
  }
  if (fin) {
    k.done = 1;
    atomicAdd(&glob->ndone, 1);
  }
}

// MIXED inner iteration: BETA = r.z / r.z_old and the inner stop test on r.r
// (its target, ITERM, or cap_fac*ITERM + 50 inner iterations over all passes).
__device__ __forceinline__ void mx_update_epi(Ctl &k, Glob *glob, int iterm, double rz, double rr,
                                              double cap_fac, int no_stop) {
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
                          k.iter >= int(cap_fac * iterm) + 50)) {
    k.idone = 1;
    atomicAdd(&glob->nidone, 1);
  } else {
    k.parity ^= 1;
  }
}

// The member-reduce kernels: member m (one CTA per member, grid-stride) sums
// its quads' partials of each of the NS sums in fixed order and, unless
// skip(m), epi(m, r) finishes it (r valid in thread 0).
template <int NS, class Skip, class Epi>
__device__ __forceinline__ void member_reduce(const DevStatic &S, const double *part, Skip skip,
                                              Epi epi) {
  __shared__ double sh[32];
  for (int m = blockIdx.x; m < S.nmember; m += gridDim.x) {
    if (skip(m)) continue;  // uniform
    const int q0 = S.qstart[m], nq = S.qstart[m + 1] - q0;
    double r[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) r[s] = reduce_partials<>(part + size_t(s) * S.nquad + q0, nq, sh);
    epi(m, r);
  }
}

// The same loop without reductions (member-wise vector updates).
template <class Skip, class Body>
__device__ __forceinline__ void quad_apply(const DevStatic &S, Skip skip, Body body) {
  const int sub = threadIdx.x / TPT, q = threadIdx.x % TPT;
  for (int qd = blockIdx.x; qd < S.nquad; qd += gridDim.x) {
    const int4 cur = S.quads[qd];
    const int m = cur.x;
    if (skip(m)) continue;
    if (sub >= cur.z) continue;
    body(m, row_geo(S.tnbr, cur.y + sub, q));
  }
}

// PCG = CCCI*RCG + BETA*PCG (congrad.f90:133-159) on the cell's row vector and
// its N/S rows and E/W neighbours, then APCG = CCC*P + CCS*PS + CCN*PN + CCW*PW
// + CCE*PE (congrad.f90:114).  Stores p_new and Ap; returns the cell part of
// p.Ap.  With asym == false, CCN(L) = CCS(LN) and CCE(L) = CCW(LE).
template <class T>
__device__ __forceinline__ double matvec_row(const RowGeo &g, bool valid, const T *__restrict__ r,
                                             const T *__restrict__ ccc,
                                             const T *__restrict__ pold, T *__restrict__ pnew,
                                             const T *__restrict__ ccs, const T *__restrict__ ccw,
                                             const T *__restrict__ cce, const T *__restrict__ ccn,
                                             T *__restrict__ ap, T beta, bool asym) {
  const V4<T> r0 = ld4(r + g.d0), c0 = ld4(ccc + g.d0), o0 = ld4(pold + g.d0);
  const V4<T> rn = ld4(r + g.dn), cn_ = ld4(ccc + g.dn), on = ld4(pold + g.dn);
  const V4<T> rs = ld4(r + g.ds), cs_ = ld4(ccc + g.ds), os = ld4(pold + g.ds);
  auto pc = [&](T rr, T cc, T po) { return rcpT(cc) * rr + beta * po; };
  const V4<T> p = {pc(r0.x, c0.x, o0.x), pc(r0.y, c0.y, o0.y), pc(r0.z, c0.z, o0.z),
                   pc(r0.w, c0.w, o0.w)};
  const V4<T> pn = {pc(rn.x, cn_.x, on.x), pc(rn.y, cn_.y, on.y), pc(rn.z, cn_.z, on.z),
                    pc(rn.w, cn_.w, on.w)};
  const V4<T> ps = {pc(rs.x, cs_.x, os.x), pc(rs.y, cs_.y, os.y), pc(rs.z, cs_.z, os.z),
                    pc(rs.w, cs_.w, os.w)};
  T pw = from_west(p), pe = from_east(p);
  if (g.cx == 0) pw = pc(r[g.dwe], ccc[g.dwe], pold[g.dwe]);
  if (g.cx == ROWT - 1) pe = pc(r[g.dee], ccc[g.dee], pold[g.dee]);
  const V4<T> ks = ld4(ccs + g.d0), kw = ld4(ccw + g.d0);
  V4<T> kn, ke;
  if (asym) {
    kn = ld4(ccn + g.d0);
    ke = ld4(cce + g.d0);
  } else {
    kn = ld4(ccs + g.dn);
    T kwe = from_east(kw);
    if (g.cx == ROWT - 1) kwe = ccw[g.dee];
    ke = {kw.y, kw.z, kw.w, kwe};
  }
  V4<T> a;
  a.x = c0.x * p.x + ks.x * ps.x + kn.x * pn.x + kw.x * pw + ke.x * p.y;
  a.y = c0.y * p.y + ks.y * ps.y + kn.y * pn.y + kw.y * p.x + ke.y * p.z;
  a.z = c0.z * p.z + ks.z * ps.z + kn.z * pn.z + kw.z * p.y + ke.z * p.w;
  a.w = c0.w * p.w + ks.w * ps.w + kn.w * pn.w + kw.w * p.z + ke.w * pe;
  if (!valid) return 0.0;
  st4(pnew + g.d0, p);
  st4(ap + g.d0, a);
  return double(a.x) * double(p.x) + double(a.y) * double(p.y) + double(a.z) * double(p.z) +
         double(a.w) * double(p.w);
}


// FP64: as matvec_row, with z = CCCI*r stored by the kernels that write r, so
// that the halo rows need z and p_old only: p = z + beta*p_old has the same
// roundings as CCCI*r + beta*p_old formed in place.  With x and dox, also the
// previous iteration's x += alpha*p_old, the statement the update pass would
// have run (same operands, same rounding): that pass then reads neither x nor
// p, and the last iteration's term is applied after the loop (k_cg_finish).
__device__ __forceinline__ double matvec_row_z(const RowGeo &g, bool valid,
                                               const double *__restrict__ z,
                                               const double *__restrict__ ccc,
                                               const double *__restrict__ pold,
                                               double *__restrict__ pnew,
                                               const double *__restrict__ ccs,
                                               const double *__restrict__ ccw,
                                               const double *__restrict__ cce,
                                               const double *__restrict__ ccn,
                                               double *__restrict__ ap, double beta, bool asym,
                                               double *__restrict__ x = nullptr,
                                               double alpha_prev = 0., bool dox = false) {
  const V4<double> z0 = ld4(z + g.d0), o0 = ld4(pold + g.d0);
  const V4<double> x0 = (x && dox) ? ld4(x + g.d0) : V4<double>{0., 0., 0., 0.};
  const V4<double> zn = ld4(z + g.dn), on = ld4(pold + g.dn);
  const V4<double> zs = ld4(z + g.ds), os = ld4(pold + g.ds);
  auto pc = [&](double zz, double po) { return zz + beta * po; };
  const V4<double> p = {pc(z0.x, o0.x), pc(z0.y, o0.y), pc(z0.z, o0.z), pc(z0.w, o0.w)};
  const V4<double> pn = {pc(zn.x, on.x), pc(zn.y, on.y), pc(zn.z, on.z), pc(zn.w, on.w)};
  const V4<double> ps = {pc(zs.x, os.x), pc(zs.y, os.y), pc(zs.z, os.z), pc(zs.w, os.w)};
  double pw = from_west(p), pe = from_east(p);
  if (g.cx == 0) pw = pc(z[g.dwe], pold[g.dwe]);
  if (g.cx == ROWT - 1) pe = pc(z[g.dee], pold[g.dee]);
  const V4<double> c0 = ld4(ccc + g.d0), ks = ld4(ccs + g.d0), kw = ld4(ccw + g.d0);
  V4<double> kn, ke;
  if (asym) {
    kn = ld4(ccn + g.d0);
    ke = ld4(cce + g.d0);
  } else {
    kn = ld4(ccs + g.dn);
    double kwe = from_east(kw);
    if (g.cx == ROWT - 1) kwe = ccw[g.dee];
    ke = {kw.y, kw.z, kw.w, kwe};
  }
  V4<double> a;
  a.x = c0.x * p.x + ks.x * ps.x + kn.x * pn.x + kw.x * pw + ke.x * p.y;
  a.y = c0.y * p.y + ks.y * ps.y + kn.y * pn.y + kw.y * p.x + ke.y * p.z;
  a.z = c0.z * p.z + ks.z * ps.z + kn.z * pn.z + kw.z * p.y + ke.z * p.w;
  a.w = c0.w * p.w + ks.w * ps.w + kn.w * pn.w + kw.w * p.z + ke.w * pe;
  if (!valid) return 0.0;
  if (x && dox)  // the previous iteration's X = X + ALPHA*PCG (congrad.f90:133)
    st4(x + g.d0, V4<double>{x0.x + alpha_prev * o0.x, x0.y + alpha_prev * o0.y,
                             x0.z + alpha_prev * o0.z, x0.w + alpha_prev * o0.w});
  st4(pnew + g.d0, p);
  st4(ap + g.d0, a);
  return a.x * p.x + a.y * p.y + a.z * p.z + a.w * p.w;
}

// MIXED inner iteration: x += alpha*p of the previous iteration, which the
// next matrix-vector pass applies (its p_old is that p, already loaded), so
// that the update pass reads neither x nor p; the last iteration's term is
// applied with the correction (k_mx_apply).  The same fmaf on the same
// values as in the update pass, hence the same x.
__device__ __forceinline__ V4<float> x_plus_alpha_p(const V4<float> &x, float alpha,
                                                    const V4<float> &p) {
  return {fmaf(alpha, p.x, x.x), fmaf(alpha, p.y, x.y), fmaf(alpha, p.z, x.z),
          fmaf(alpha, p.w, x.w)};
}

// MIXED inner CG on the Jacobi-scaled system (unit diagonal): p = r + beta*p
// at the row vector and its halo, Ap = p + AS*pS + AN*pN + AW*pW + AE*pE, and
// the part of p.Ap.  Symmetric: AN(L) = AS(LN), AE(L) = AW(LE).  With dox,
// also the previous iteration's x += alpha*p (x_plus_alpha_p).
__device__ __forceinline__ double matvec_row_scaled(const RowGeo &g, bool valid,
                                                    const float *__restrict__ r,
                                                    const float *__restrict__ pold,
                                                    float *__restrict__ pnew,
                                                    const float *__restrict__ as,
                                                    const float *__restrict__ aw,
                                                    const float *__restrict__ ae,
                                                    const float *__restrict__ an,
                                                    float *__restrict__ ap, float beta, bool asym,
                                                    float *__restrict__ x, float alpha_prev,
                                                    bool dox) {
  const V4<float> r0 = ld4(r + g.d0), o0 = ld4(pold + g.d0);
  const V4<float> x0 = dox ? ld4(x + g.d0) : V4<float>{0.f, 0.f, 0.f, 0.f};
  const V4<float> rn = ld4(r + g.dn), on = ld4(pold + g.dn);
  const V4<float> rs = ld4(r + g.ds), os = ld4(pold + g.ds);
  const V4<float> p = {fmaf(beta, o0.x, r0.x), fmaf(beta, o0.y, r0.y), fmaf(beta, o0.z, r0.z),
                       fmaf(beta, o0.w, r0.w)};
  const V4<float> pn = {fmaf(beta, on.x, rn.x), fmaf(beta, on.y, rn.y), fmaf(beta, on.z, rn.z),
                        fmaf(beta, on.w, rn.w)};
  const V4<float> ps = {fmaf(beta, os.x, rs.x), fmaf(beta, os.y, rs.y), fmaf(beta, os.z, rs.z),
                        fmaf(beta, os.w, rs.w)};
  float pw = from_west(p), pe = from_east(p);
  if (g.cx == 0) pw = fmaf(beta, pold[g.dwe], r[g.dwe]);
  if (g.cx == ROWT - 1) pe = fmaf(beta, pold[g.dee], r[g.dee]);
  const V4<float> ks = ld4(as + g.d0), kw = ld4(aw + g.d0);
  V4<float> kn, ke;
  if (asym) {
    kn = ld4(an + g.d0);
    ke = ld4(ae + g.d0);
  } else {
    kn = ld4(as + g.dn);
    float kwe = from_east(kw);
    if (g.cx == ROWT - 1) kwe = aw[g.dee];
    ke = {kw.y, kw.z, kw.w, kwe};
  }
  V4<float> a;
  a.x = p.x + ks.x * ps.x + kn.x * pn.x + kw.x * pw + ke.x * p.y;
  a.y = p.y + ks.y * ps.y + kn.y * pn.y + kw.y * p.x + ke.y * p.z;
  a.z = p.z + ks.z * ps.z + kn.z * pn.z + kw.z * p.y + ke.z * p.w;
  a.w = p.w + ks.w * ps.w + kn.w * pn.w + kw.w * p.z + ke.w * pe;
  if (!valid) return 0.0;
  if (dox) st4(x + g.d0, x_plus_alpha_p(x0, alpha_prev, o0));
  st4(pnew + g.d0, p);
  st4(ap + g.d0, a);
  return double(a.x) * double(p.x) + double(a.y) * double(p.y) + double(a.z) * double(p.z) +
         double(a.w) * double(p.w);
}

// MIXED, polynomial-preconditioned: r -= alpha*Ap at the cell
// and (recomputed from r and Ap) at its four neighbours, then
// z = (2I - Ahat) r = r - N r (N: the couplings AS, AW, AN = AS(LN),
// AE = AW(LE)) -- the two-term Neumann series of Ahat^-1, symmetric positive
// definite for a symmetric unit-diagonal Ahat with eigenvalues in (0, 2).
// With poly == false z = r (Jacobi; unsymmetric operators).  Stores the new
// r (into the other residual buffer: neighbours still read the old r for
// their own halo) and z; adds r.z and r.r.  (x += alpha*p: the next
// matrix-vector pass, x_plus_alpha_p.)
__device__ __forceinline__ void update_row_poly(const RowGeo &g, bool valid,
                                                const float *__restrict__ r,
                                                float *__restrict__ rnew,
                                                const float *__restrict__ ap,
                                                const float *__restrict__ as,
                                                const float *__restrict__ aw,
                                                float *__restrict__ z, float alpha, bool poly,
                                                double &rz, double &rr) {
  const V4<float> r0 = ld4(r + g.d0), a0 = ld4(ap + g.d0);
  const V4<float> rn0 = {fmaf(-alpha, a0.x, r0.x), fmaf(-alpha, a0.y, r0.y),
                         fmaf(-alpha, a0.z, r0.z), fmaf(-alpha, a0.w, r0.w)};
  V4<float> zv = rn0;
  if (poly) {
    const V4<float> rN = ld4(r + g.dn), aN = ld4(ap + g.dn);
    const V4<float> rS = ld4(r + g.ds), aS = ld4(ap + g.ds);
    const V4<float> nN = {fmaf(-alpha, aN.x, rN.x), fmaf(-alpha, aN.y, rN.y),
                          fmaf(-alpha, aN.z, rN.z), fmaf(-alpha, aN.w, rN.w)};
    const V4<float> nS = {fmaf(-alpha, aS.x, rS.x), fmaf(-alpha, aS.y, rS.y),
                          fmaf(-alpha, aS.z, rS.z), fmaf(-alpha, aS.w, rS.w)};
    float nw = from_west(rn0), ne = from_east(rn0);
    if (g.cx == 0) nw = fmaf(-alpha, ap[g.dwe], r[g.dwe]);
    if (g.cx == ROWT - 1) ne = fmaf(-alpha, ap[g.dee], r[g.dee]);
    const V4<float> ks = ld4(as + g.d0), kw = ld4(aw + g.d0), kn = ld4(as + g.dn);
    float kwe = from_east(kw);
    if (g.cx == ROWT - 1) kwe = aw[g.dee];
    const V4<float> ke = {kw.y, kw.z, kw.w, kwe};
    zv.x = rn0.x - (ks.x * nS.x + kn.x * nN.x + kw.x * nw + ke.x * rn0.y);
    zv.y = rn0.y - (ks.y * nS.y + kn.y * nN.y + kw.y * rn0.x + ke.y * rn0.z);
    zv.z = rn0.z - (ks.z * nS.z + kn.z * nN.z + kw.z * rn0.y + ke.z * rn0.w);
    zv.w = rn0.w - (ks.w * nS.w + kn.w * nN.w + kw.w * rn0.z + ke.w * ne);
  }
  if (!valid) return;
  st4(rnew + g.d0, rn0);
  st4(z + g.d0, zv);
  rz += double(rn0.x) * double(zv.x) + double(rn0.y) * double(zv.y) +
        double(rn0.z) * double(zv.z) + double(rn0.w) * double(zv.w);
  rr += double(rn0.x) * double(rn0.x) + double(rn0.y) * double(rn0.y) +
        double(rn0.z) * double(rn0.z) + double(rn0.w) * double(rn0.w);
}

// MIXED: z0 = (2I - Ahat) r (or r) for the first inner iteration, p_old = 0,
// and the part of r.z.
__device__ __forceinline__ double zinit_row(const RowGeo &g, bool valid,
                                           const float *__restrict__ r,
                                           const float *__restrict__ as,
                                           const float *__restrict__ aw, float *__restrict__ z,
                                           float *__restrict__ pold, bool poly) {
  const V4<float> r0 = ld4(r + g.d0);
  V4<float> zv = r0;
  if (poly) {
    const V4<float> rN = ld4(r + g.dn), rS = ld4(r + g.ds);
    float rw = from_west(r0), re = from_east(r0);
    if (g.cx == 0) rw = r[g.dwe];
    if (g.cx == ROWT - 1) re = r[g.dee];
    const V4<float> ks = ld4(as + g.d0), kw = ld4(aw + g.d0), kn = ld4(as + g.dn);
    float kwe = from_east(kw);
    if (g.cx == ROWT - 1) kwe = aw[g.dee];
    const V4<float> ke = {kw.y, kw.z, kw.w, kwe};
    zv.x = r0.x - (ks.x * rS.x + kn.x * rN.x + kw.x * rw + ke.x * r0.y);
    zv.y = r0.y - (ks.y * rS.y + kn.y * rN.y + kw.y * r0.x + ke.y * r0.z);
    zv.z = r0.z - (ks.z * rS.z + kn.z * rN.z + kw.z * r0.y + ke.z * r0.w);
    zv.w = r0.w - (ks.w * rS.w + kn.w * rN.w + kw.w * r0.z + ke.w * re);
  }
  if (!valid) return 0.0;
  st4(z + g.d0, zv);
  st4(pold + g.d0, V4<float>{0.f, 0.f, 0.f, 0.f});
  return double(r0.x) * double(zv.x) + double(r0.y) * double(zv.y) + double(r0.z) * double(zv.z) +
         double(r0.w) * double(zv.w);
}

// Variant 3 of the MIXED inner iteration: matvec_row_scaled and
// update_row_poly with every global load of the row issued before the first
// shuffle or dependent operation (above, the coefficient rows and x, p_new
// wait for the first loads' values), so that one round trip to memory serves
// the row; the same operations on the same values, hence the same results.
// It holds more values live: its kernels run at fewer CTAs per SM.
__device__ __forceinline__ double matvec_row_scaled_eager(const RowGeo &g, bool valid,
                                                    const float *__restrict__ r,
                                                    const float *__restrict__ pold,
                                                    float *__restrict__ pnew,
                                                    const float *__restrict__ as,
                                                    const float *__restrict__ aw,
                                                    const float *__restrict__ ae,
                                                    const float *__restrict__ an,
                                                    float *__restrict__ ap, float beta, bool asym,
                                                    float *__restrict__ x, float alpha_prev,
                                                    bool dox) {
  // every load first, so that one round trip serves the row (x is read at
  // the ghost tile's inert slots too when the row is not valid)
  const V4<float> r0 = ld4(r + g.d0), o0 = ld4(pold + g.d0);
  const V4<float> x0 = dox ? ld4(x + g.d0) : V4<float>{0.f, 0.f, 0.f, 0.f};
  const V4<float> rn = ld4(r + g.dn), on = ld4(pold + g.dn);
  const V4<float> rs = ld4(r + g.ds), os = ld4(pold + g.ds);
  const V4<float> ks = ld4(as + g.d0), kw = ld4(aw + g.d0);
  const V4<float> kn = asym ? ld4(an + g.d0) : ld4(as + g.dn);
  V4<float> ke = asym ? ld4(ae + g.d0) : V4<float>{0.f, 0.f, 0.f, 0.f};
  const bool west = g.cx == 0, east = g.cx == ROWT - 1;
  const float rw = west ? r[g.dwe] : 0.f, ow = west ? pold[g.dwe] : 0.f;
  const float re = east ? r[g.dee] : 0.f, oe = east ? pold[g.dee] : 0.f;
  const float kwe_edge = (east && !asym) ? aw[g.dee] : 0.f;
  const V4<float> p = {fmaf(beta, o0.x, r0.x), fmaf(beta, o0.y, r0.y), fmaf(beta, o0.z, r0.z),
                       fmaf(beta, o0.w, r0.w)};
  const V4<float> pn = {fmaf(beta, on.x, rn.x), fmaf(beta, on.y, rn.y), fmaf(beta, on.z, rn.z),
                        fmaf(beta, on.w, rn.w)};
  const V4<float> ps = {fmaf(beta, os.x, rs.x), fmaf(beta, os.y, rs.y), fmaf(beta, os.z, rs.z),
                        fmaf(beta, os.w, rs.w)};
  float pw = from_west(p), pe = from_east(p);
  if (west) pw = fmaf(beta, ow, rw);
  if (east) pe = fmaf(beta, oe, re);
  if (!asym) {
    float kwe = from_east(kw);
    if (east) kwe = kwe_edge;
    ke = {kw.y, kw.z, kw.w, kwe};
  }
  V4<float> a;
  a.x = p.x + ks.x * ps.x + kn.x * pn.x + kw.x * pw + ke.x * p.y;
  a.y = p.y + ks.y * ps.y + kn.y * pn.y + kw.y * p.x + ke.y * p.z;
  a.z = p.z + ks.z * ps.z + kn.z * pn.z + kw.z * p.y + ke.z * p.w;
  a.w = p.w + ks.w * ps.w + kn.w * pn.w + kw.w * p.z + ke.w * pe;
  if (!valid) return 0.0;
  if (dox) st4(x + g.d0, x_plus_alpha_p(x0, alpha_prev, o0));
  st4(pnew + g.d0, p);
  st4(ap + g.d0, a);
  return double(a.x) * double(p.x) + double(a.y) * double(p.y) + double(a.z) * double(p.z) +
         double(a.w) * double(p.w);
}

__device__ __forceinline__ void update_row_poly_eager(const RowGeo &g, bool valid,
                                                const float *__restrict__ r,
                                                float *__restrict__ rnew,
                                                const float *__restrict__ ap,
                                                const float *__restrict__ as,
                                                const float *__restrict__ aw,
                                                float *__restrict__ z, float alpha, bool poly,
                                                double &rz, double &rr) {
  // every load first, so that one round trip serves the row
  const V4<float> r0 = ld4(r + g.d0), a0 = ld4(ap + g.d0);
  V4<float> rN{}, aN{}, rS{}, aS{}, ks{}, kw{}, kn{};
  float rw = 0.f, aw_ = 0.f, re = 0.f, ae_ = 0.f, kwe_edge = 0.f;
  const bool west = g.cx == 0, east = g.cx == ROWT - 1;
  if (poly) {
    rN = ld4(r + g.dn);
    aN = ld4(ap + g.dn);
    rS = ld4(r + g.ds);
    aS = ld4(ap + g.ds);
    ks = ld4(as + g.d0);
    kw = ld4(aw + g.d0);
    kn = ld4(as + g.dn);
    if (west) {
      rw = r[g.dwe];
      aw_ = ap[g.dwe];
    }
    if (east) {
      re = r[g.dee];
      ae_ = ap[g.dee];
      kwe_edge = aw[g.dee];
    }
  }
  const V4<float> rn0 = {fmaf(-alpha, a0.x, r0.x), fmaf(-alpha, a0.y, r0.y),
                         fmaf(-alpha, a0.z, r0.z), fmaf(-alpha, a0.w, r0.w)};
  V4<float> zv = rn0;
  if (poly) {
    const V4<float> nN = {fmaf(-alpha, aN.x, rN.x), fmaf(-alpha, aN.y, rN.y),
                          fmaf(-alpha, aN.z, rN.z), fmaf(-alpha, aN.w, rN.w)};
    const V4<float> nS = {fmaf(-alpha, aS.x, rS.x), fmaf(-alpha, aS.y, rS.y),
                          fmaf(-alpha, aS.z, rS.z), fmaf(-alpha, aS.w, rS.w)};
    float nw = from_west(rn0), ne = from_east(rn0);
    if (west) nw = fmaf(-alpha, aw_, rw);
    if (east) ne = fmaf(-alpha, ae_, re);
    float kwe = from_east(kw);
    if (east) kwe = kwe_edge;
    const V4<float> ke = {kw.y, kw.z, kw.w, kwe};
    zv.x = rn0.x - (ks.x * nS.x + kn.x * nN.x + kw.x * nw + ke.x * rn0.y);
    zv.y = rn0.y - (ks.y * nS.y + kn.y * nN.y + kw.y * rn0.x + ke.y * rn0.z);
    zv.z = rn0.z - (ks.z * nS.z + kn.z * nN.z + kw.z * rn0.y + ke.z * rn0.w);
    zv.w = rn0.w - (ks.w * nS.w + kn.w * nN.w + kw.w * rn0.z + ke.w * ne);
  }
  if (!valid) return;
  st4(rnew + g.d0, rn0);
  st4(z + g.d0, zv);
  rz += double(rn0.x) * double(zv.x) + double(rn0.y) * double(zv.y) +
        double(rn0.z) * double(zv.z) + double(rn0.w) * double(zv.w);
  rr += double(rn0.x) * double(rn0.x) + double(rn0.y) * double(rn0.y) +
        double(rn0.z) * double(rn0.z) + double(rn0.w) * double(rn0.w);
}

// MIXED, Jacobi: r -= alpha*Ap (into the other residual buffer) and the part
// of r.r (= r.z on the unit-diagonal system).  (x += alpha*p: the next
// matrix-vector pass, x_plus_alpha_p.)
__device__ __forceinline__ void update_row_jac(const RowGeo &g, bool valid,
                                               const float *__restrict__ r,
                                               float *__restrict__ rnew,
                                               const float *__restrict__ ap, float alpha,
                                               double &rr) {
  if (!valid) return;
  V4<float> rv = ld4(r + g.d0);
  const V4<float> av = ld4(ap + g.d0);
  rv.x = fmaf(-alpha, av.x, rv.x);
  rv.y = fmaf(-alpha, av.y, rv.y);
  rv.z = fmaf(-alpha, av.z, rv.z);
  rv.w = fmaf(-alpha, av.w, rv.w);
  st4(rnew + g.d0, rv);
  rr += double(rv.x) * double(rv.x) + double(rv.y) * double(rv.y) + double(rv.z) * double(rv.z) +
        double(rv.w) * double(rv.w);
}

// X = X + ALPHA*PCG, RCG = RCG - ALPHA*APCG, TMPCG = CCCI*RCG (congrad.f90:
// 133-135) and the parts of r.z and r.r (:143-146).
template <class T>
__device__ __forceinline__ void update_row(const RowGeo &g, bool valid, T *__restrict__ x,
                                           const T *__restrict__ pnew, T *__restrict__ r,
                                           const T *__restrict__ ap, const T *__restrict__ ccc,
                                           T alpha, double &rz, double &rr,
                                           T *__restrict__ zout = nullptr) {
  if (!valid) return;
  V4<T> rv = ld4(r + g.d0);
  const V4<T> av = ld4(ap + g.d0), cv = ld4(ccc + g.d0);
  if (x) {  // (nullptr: the next matrix-vector pass adds alpha*p, matvec_row_z)
    V4<T> xv = ld4(x + g.d0);
    const V4<T> pv = ld4(pnew + g.d0);
    xv.x = xv.x + alpha * pv.x;
    xv.y = xv.y + alpha * pv.y;
    xv.z = xv.z + alpha * pv.z;
    xv.w = xv.w + alpha * pv.w;
    st4(x + g.d0, xv);
  }
  rv.x = rv.x - alpha * av.x;
  rv.y = rv.y - alpha * av.y;
  rv.z = rv.z - alpha * av.z;
  rv.w = rv.w - alpha * av.w;
  st4(r + g.d0, rv);
  const T z0 = rcpT(cv.x) * rv.x, z1 = rcpT(cv.y) * rv.y, z2 = rcpT(cv.z) * rv.z,
          z3 = rcpT(cv.w) * rv.w;
  if (zout) st4(zout + g.d0, V4<T>{z0, z1, z2, z3});
  rz += double(rv.x) * double(z0) + double(rv.y) * double(z1) + double(rv.z) * double(z2) +
        double(rv.w) * double(z3);
  rr += double(rv.x) * double(rv.x) + double(rv.y) * double(rv.y) + double(rv.z) * double(rv.z) +
        double(rv.w) * double(rv.w);
}

// RCG = FPTMP - CCC*P - CCN*PN - CCS*PS - CCW*PW - CCE*PE (congrad.f90:72) in
// FP64 on a row vector of the system V; land slots give 0.
__device__ __forceinline__ V4<double> residual_row(const RowGeo &g, const uint8_t *kind,
                                                   const double *__restrict__ P,
                                                   const SysView &V, bool asym) {
  const V4<double> x = ld4(P + g.d0), xn = ld4(P + g.dn), xs = ld4(P + g.ds);
  double xw = from_west(x), xe = from_east(x);
  if (g.cx == 0) xw = P[g.dwe];
  if (g.cx == ROWT - 1) xe = P[g.dee];
  const V4<double> b = ld4(V.fp + g.d0), c = ld4(V.cc + g.d0), ks = ld4(V.cs + g.d0),
                   kw = ld4(V.cw + g.d0);
  V4<double> kn, ke;
  if (asym) {
    kn = ld4(V.cn + g.d0);
    ke = ld4(V.ce + g.d0);
  } else {  // CCN(L) = CCS(LN), CCE(L) = CCW(LE)
    kn = ld4(V.cs + g.dn);
    double kwe = from_east(kw);
    if (g.cx == ROWT - 1) kwe = V.cw[g.dee];
    ke = {kw.y, kw.z, kw.w, kwe};
  }
  const uchar4 kd = *reinterpret_cast<const uchar4 *>(kind + g.d0);
  V4<double> r;
  r.x = b.x - c.x * x.x - kn.x * xn.x - ks.x * xs.x - kw.x * xw - ke.x * x.y;
  r.y = b.y - c.y * x.y - kn.y * xn.y - ks.y * xs.y - kw.y * x.x - ke.y * x.z;
  r.z = b.z - c.z * x.z - kn.z * xn.z - ks.z * xs.z - kw.z * x.y - ke.z * x.w;
  r.w = b.w - c.w * x.w - kn.w * xn.w - ks.w * xs.w - kw.w * x.z - ke.w * xe;
  if (kd.x == LAND) r.x = 0.;
  if (kd.y == LAND) r.y = 0.;
  if (kd.z == LAND) r.z = 0.;
  if (kd.w == LAND) r.w = 0.;
  return r;
}

__device__ __forceinline__ V4<double> residual_row(const RowGeo &g, const uint8_t *kind,
                                                   const double *__restrict__ P,
                                                   const DevSystem &Y, bool asym) {
  return residual_row(g, kind, P, SysView{Y.fptmp, Y.ccc, Y.ccs, Y.ccw, Y.cce, Y.ccn, 0}, asym);
}

// residual_row and zinit_row with every load of the row issued first (the
// refinement kernels of variant 3, see matvec_row_scaled_eager).
__device__ __forceinline__ V4<double> residual_row_eager(const RowGeo &g, const uint8_t *kind,
                                                   const double *__restrict__ P,
                                                   const SysView &V, bool asym) {
  // every load first, so that one round trip serves the row
  const V4<double> x = ld4(P + g.d0), xn = ld4(P + g.dn), xs = ld4(P + g.ds);
  const V4<double> b = ld4(V.fp + g.d0), c = ld4(V.cc + g.d0), ks = ld4(V.cs + g.d0),
                   kw = ld4(V.cw + g.d0);
  const V4<double> kn = asym ? ld4(V.cn + g.d0) : ld4(V.cs + g.dn);  // CCN(L) = CCS(LN)
  V4<double> ke = asym ? ld4(V.ce + g.d0) : V4<double>{0., 0., 0., 0.};
  const uchar4 kd = *reinterpret_cast<const uchar4 *>(kind + g.d0);
  const bool west = g.cx == 0, east = g.cx == ROWT - 1;
  const double xw_edge = west ? P[g.dwe] : 0., xe_edge = east ? P[g.dee] : 0.;
  const double kwe_edge = (east && !asym) ? V.cw[g.dee] : 0.;
  double xw = from_west(x), xe = from_east(x);
  if (west) xw = xw_edge;
  if (east) xe = xe_edge;
  if (!asym) {  // CCE(L) = CCW(LE)
    double kwe = from_east(kw);
    if (east) kwe = kwe_edge;
    ke = {kw.y, kw.z, kw.w, kwe};
  }
  V4<double> r;
  r.x = b.x - c.x * x.x - kn.x * xn.x - ks.x * xs.x - kw.x * xw - ke.x * x.y;
  r.y = b.y - c.y * x.y - kn.y * xn.y - ks.y * xs.y - kw.y * x.x - ke.y * x.z;
  r.z = b.z - c.z * x.z - kn.z * xn.z - ks.z * xs.z - kw.z * x.y - ke.z * x.w;
  r.w = b.w - c.w * x.w - kn.w * xn.w - ks.w * xs.w - kw.w * x.z - ke.w * xe;
  if (kd.x == LAND) r.x = 0.;
  if (kd.y == LAND) r.y = 0.;
  if (kd.z == LAND) r.z = 0.;
  if (kd.w == LAND) r.w = 0.;
  return r;
}

__device__ __forceinline__ double zinit_row_eager(const RowGeo &g, bool valid,
                                           const float *__restrict__ r,
                                           const float *__restrict__ as,
                                           const float *__restrict__ aw, float *__restrict__ z,
                                           float *__restrict__ pold, bool poly) {
  // every load first, so that one round trip serves the row
  const V4<float> r0 = ld4(r + g.d0);
  V4<float> rN{}, rS{}, ks{}, kw{}, kn{};
  float rw_edge = 0.f, re_edge = 0.f, kwe_edge = 0.f;
  const bool west = g.cx == 0, east = g.cx == ROWT - 1;
  if (poly) {
    rN = ld4(r + g.dn);
    rS = ld4(r + g.ds);
    ks = ld4(as + g.d0);
    kw = ld4(aw + g.d0);
    kn = ld4(as + g.dn);
    if (west) rw_edge = r[g.dwe];
    if (east) {
      re_edge = r[g.dee];
      kwe_edge = aw[g.dee];
    }
  }
  V4<float> zv = r0;
  if (poly) {
    float rw = from_west(r0), re = from_east(r0);
    if (west) rw = rw_edge;
    if (east) re = re_edge;
    float kwe = from_east(kw);
    if (east) kwe = kwe_edge;
    const V4<float> ke = {kw.y, kw.z, kw.w, kwe};
    zv.x = r0.x - (ks.x * rS.x + kn.x * rN.x + kw.x * rw + ke.x * r0.y);
    zv.y = r0.y - (ks.y * rS.y + kn.y * rN.y + kw.y * r0.x + ke.y * r0.z);
    zv.z = r0.z - (ks.z * rS.z + kn.z * rN.z + kw.z * r0.y + ke.z * r0.w);
    zv.w = r0.w - (ks.w * rS.w + kn.w * rN.w + kw.w * r0.z + ke.w * re);
  }
  if (!valid) return 0.0;
  st4(z + g.d0, zv);
  st4(pold + g.d0, V4<float>{0.f, 0.f, 0.f, 0.f});
  return double(r0.x) * double(zv.x) + double(r0.y) * double(zv.y) + double(r0.z) * double(zv.z) +
         double(r0.w) * double(zv.w);
}

// The Jacobi scaling of the MIXED inner system, 1/sqrt(c) for a diagonal c
// (0 where c <= 0: land slots of an unscaled system): the FP32 hardware
// estimate refined by one Newton-Raphson step y(3 - c y^2)/2 in FP64
// (relative error ~1e-13).  Explicitly rounded operations, so every kernel
// (whatever its contraction flags) gets the same value for the same c: the
// operator, the scaled residual and the correction all use one D.
__device__ __forceinline__ double inv_sqrt_diag(double c) {
  if (!(c > 0.0)) return 0.0;
  const double y = double(rsqrtf(float(c)));
  const double t = __dmul_rn(__dmul_rn(c, y), y);
  return __dmul_rn(y, __fma_rn(-0.5, t, 1.5));
}

}  // namespace xm
