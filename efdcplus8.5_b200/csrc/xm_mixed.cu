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

#include <map>
#include <mutex>

#include "xm_cg.cuh"
#include "xm_kernels.h"

namespace xm {

#define TILE_LOOP(ntile)                                                      \
  for (int tile = blockIdx.x + 1; tile < (ntile); tile += gridDim.x)

// p = z + beta*p_old at the cell and its halo (z = r for Jacobi members),
// Ahat*p, p.Ap (per member).
// CTAs per SM the launch bounds ask for, by variant (3 holds more values live)
constexpr int mx_ctas(int var) { return var == 1 ? 5 : var == 3 ? 4 : 6; }
// variant 3's matrix-vector and update kernels (measured on the 256-member
// ensemble: 3 for the first, no spills at 72 registers, is even; 5 for the
// second spills and is 3 % slower)
constexpr int MV3_CTAS = 4, UP3_CTAS = 4;
constexpr int mv_ctas(int var) { return var == 3 ? MV3_CTAS : mx_ctas(var); }
constexpr int up_ctas(int var) { return var == 3 ? UP3_CTAS : mx_ctas(var); }

template <bool MA, int VAR, bool FOLD>
__global__ void __launch_bounds__(NT, mv_ctas(VAR)) k_mx_matvec(DevStatic S, DevSystem Y, Ctl *ctl,
                                                    double *part) {
  struct A {
    bool skip, asym, dox;
    float beta, alpha;
    const float *pold;
    float *pnew;
    const float *z;
  };
  quad_sweep_v<1, VAR>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        const bool asym = unsym<MA>(k);
        const bool poly = Y.mpoly[m] && !asym;
        // after the pass's first iteration: the previous x += alpha*p, with
        // p_old that p and alpha still the previous ALPHA
        return A{(k.done | k.idone) != 0, asym, k.inner_iter > 0, float(k.beta),
                 float(k.alpha), par ? Y.pb32 : Y.pa32, par ? Y.pa32 : Y.pb32,
                 poly ? Y.z32 : (par ? Y.r32b : Y.r32)};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        if constexpr (VAR == 3)
          v[0] = matvec_row_scaled_eager(g, valid, a.z, a.pold, a.pnew, Y.as32, Y.aw32, Y.ae32,
                                         Y.an32, Y.ap32, a.beta, a.asym, Y.x32, a.alpha, a.dox);
        else
          v[0] = matvec_row_scaled(g, valid, a.z, a.pold, a.pnew, Y.as32, Y.aw32, Y.ae32,
                                   Y.an32, Y.ap32, a.beta, a.asym, Y.x32, a.alpha, a.dox);
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0) cg_matvec_epi(ctl[m], sum[0]);
      }));
}
// ALPHA = RPCG / p.Ap
__global__ void __launch_bounds__(NT) k_red_mx_matvec(DevStatic S, Ctl *ctl, const double *part) {
  member_reduce<1>(
      S, part, [&](int m) { return (ctl[m].done | ctl[m].idone) != 0; },
      [&](int m, const double *sum) {
        if (threadIdx.x == 0) cg_matvec_epi(ctl[m], sum[0]);
      });
}

// r -= alpha*Ap, z = (2I - Ahat) r (the two-term Neumann polynomial), r.z
// and r.r (FP64 sums): the members that use it.  x += alpha*p is the next
// matrix-vector kernel's (or, after the last iteration, k_mx_apply's).
template <int VAR, bool FOLD>
__global__ void __launch_bounds__(NT, up_ctas(VAR)) k_mx_update_poly(DevStatic S, DevSystem Y,
                                                         Ctl *ctl, double *part, RedArgs ra) {
  struct A {
    bool skip;
    float alpha;
    const float *r;
    float *rnew;
  };
  quad_sweep_v<2, VAR>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        const bool poly = Y.mpoly[m] && !unsym<true>(k);
        return A{(k.done | k.idone) != 0 || !poly, float(k.alpha), par ? Y.r32b : Y.r32,
                 par ? Y.r32 : Y.r32b};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        if constexpr (VAR == 3)
          update_row_poly_eager(g, valid, a.r, a.rnew, Y.ap32, Y.as32, Y.aw32, Y.z32, a.alpha,
                                true, v[0], v[1]);
        else
          update_row_poly(g, valid, a.r, a.rnew, Y.ap32, Y.as32, Y.aw32, Y.z32, a.alpha, true,
                          v[0], v[1]);
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0)
          mx_update_epi(ctl[m], ra.glob, S.sc[m].iterm, sum[0], sum[1], 2.0, ra.no_stop);
      }));
}
// The same for the Jacobi members (z = r): r and r.r only.
template <int VAR, bool FOLD>
__global__ void __launch_bounds__(NT) k_mx_update_jac(DevStatic S, DevSystem Y, Ctl *ctl,
                                                     double *part, RedArgs ra) {
  struct A {
    bool skip;
    float alpha;
    const float *r;
    float *rnew;
  };
  quad_sweep_v<2, VAR>(
      S, part,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        const bool poly = Y.mpoly[m] && !unsym<true>(k);
        return A{(k.done | k.idone) != 0 || poly, float(k.alpha), par ? Y.r32b : Y.r32,
                 par ? Y.r32 : Y.r32b};
      },
      [&](const A &a, const RowGeo &g, bool valid, double *v) {
        double rr = 0.0;
        update_row_jac(g, valid, a.r, a.rnew, Y.ap32, a.alpha, rr);
        v[0] = rr;
        v[1] = rr;
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0)
          mx_update_epi(ctl[m], ra.glob, S.sc[m].iterm, sum[0], sum[1], 2.0, ra.no_stop);
      }));
}
// BETA = r.z / r.z_old and the inner stop test on r.r.  With no_stop the
// inner solve runs past its target (kernel timing only).
__global__ void __launch_bounds__(NT) k_red_mx_update(DevStatic S, Ctl *ctl, Glob *glob,
                                                     const double *part, double total_cap_fac,
                                                     int no_stop) {
  member_reduce<2>(
      S, part, [&](int m) { return (ctl[m].done | ctl[m].idone) != 0; },
      [&](int m, const double *sum) {
        if (threadIdx.x == 0)
          mx_update_epi(ctl[m], glob, S.sc[m].iterm, sum[0], sum[1], total_cap_fac, no_stop);
      });
}

// First inner iteration of the polynomial members: z0 = (2I - Ahat) r0,
// p_old = 0, RPCG = r0.z0 (Jacobi members start from k_mx_resid's p0 = r0).
template <bool EAGER, bool FOLD>
__global__ void __launch_bounds__(NT) k_mx_zinit(DevStatic S, DevSystem Y, Ctl *ctl,
                                                double *part) {
  struct A {
    bool skip, asym;
  };
  quad_sweep<1>(
      S, part,
      [&](int m) { return A{ctl[m].done != 0 || !Y.mpoly[m] || unsym<true>(ctl[m]), false}; },
      [&](const A &, const RowGeo &g, bool valid, double *v) {
        if constexpr (EAGER)
          v[0] = zinit_row_eager(g, valid, Y.r32, Y.as32, Y.aw32, Y.z32, Y.pa32, true);
        else
          v[0] = zinit_row(g, valid, Y.r32, Y.as32, Y.aw32, Y.z32, Y.pa32, true);
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0) ctl[m].rpcg = sum[0];
      }));
}
__global__ void __launch_bounds__(NT) k_red_mx_zinit(DevStatic S, DevSystem Y, Ctl *ctl,
                                                     const double *part) {
  member_reduce<1>(
      S, part, [&](int m) { return ctl[m].done != 0 || !Y.mpoly[m] || unsym<true>(ctl[m]); },
      [&](int m, const double *sum) {
        if (threadIdx.x == 0) ctl[m].rpcg = sum[0];
      });
}


// ---------------------------------------------------------------------------
// Variant 2: the same three kernels on the staged sweep (quad_sweep_staged):
// the rows come from shared memory, filled by bulk copies one quad ahead.  The
// arithmetic is the row functions' above, operand for operand, so the results
// are those of variants 0 and 1 bit for bit.

// What a thread loads before its stage is waited for: the halo row of its
// tile's edge row (h0..h2: three arrays' N row for a row-7 thread, two arrays'
// S row for a row-0 thread) and its E/W edge values (cx == 0: the west
// neighbour of cell 0; cx == ROWT-1: the east neighbour of cell 3).
struct Halo {
  V4<float> h0, h1, h2;
  float w0, w1, e0, e1, e2;
};

constexpr int MV_STAGES = 3, POLY_STAGES = 2, JAC_STAGES = 2;
using MvStage = Stage<4>;    // z, p_old, AS, AW
using PolyStage = Stage<4>;  // r, Ap, AS, AW
using JacStage = Stage<2>;   // r, Ap

template <bool MA, bool FOLD>
__global__ void __launch_bounds__(NT, 3) k_mx_matvec_st(DevStatic S, DevSystem Y, Ctl *ctl,
                                                       double *part) {
  struct A {
    bool skip, asym, dox;
    float beta, alpha;
    float *pnew;
    const float *b[4];
  };
  quad_sweep_staged<1, 4, MV_STAGES>(
      S, part, Y.err,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        const bool asym = unsym<MA>(k);
        const bool poly = Y.mpoly[m] && !asym;
        const float *z = poly ? Y.z32 : (par ? Y.r32b : Y.r32);
        return A{(k.done | k.idone) != 0, asym, k.inner_iter > 0, float(k.beta), float(k.alpha),
                 par ? Y.pa32 : Y.pb32, {z, par ? Y.pb32 : Y.pa32, Y.as32, Y.aw32}};
      },
      [&](const A &a, const RowGeo &g, const StageRow &row) {
        Halo h{};
        if (row.north) {
          h.h0 = ld4(a.b[0] + g.dn);
          h.h1 = ld4(a.b[1] + g.dn);
          h.h2 = ld4(Y.as32 + g.dn);
        } else if (row.south) {
          h.h0 = ld4(a.b[0] + g.ds);
          h.h1 = ld4(a.b[1] + g.ds);
        }
        if (g.cx == 0) {
          h.w0 = a.b[0][g.dwe];
          h.w1 = a.b[1][g.dwe];
        }
        if (g.cx == ROWT - 1) {
          h.e0 = a.b[0][g.dee];
          h.e1 = a.b[1][g.dee];
          h.e2 = Y.aw32[g.dee];
        }
        return h;
      },
      [&](const A &a, const MvStage &st, const StageRow &row, const RowGeo &g, bool valid,
          const Halo &e, double *v) {
        const float beta = a.beta;
        const V4<float> r0 = st_body(st, 0, row), o0 = st_body(st, 1, row);
        const V4<float> rn = st_north(st, 0, row, e.h0), on = st_north(st, 1, row, e.h1);
        const V4<float> rs = st_south(st, 0, row, e.h0), os = st_south(st, 1, row, e.h1);
        const V4<float> p = {fmaf(beta, o0.x, r0.x), fmaf(beta, o0.y, r0.y),
                             fmaf(beta, o0.z, r0.z), fmaf(beta, o0.w, r0.w)};
        const V4<float> pn = {fmaf(beta, on.x, rn.x), fmaf(beta, on.y, rn.y),
                              fmaf(beta, on.z, rn.z), fmaf(beta, on.w, rn.w)};
        const V4<float> ps = {fmaf(beta, os.x, rs.x), fmaf(beta, os.y, rs.y),
                              fmaf(beta, os.z, rs.z), fmaf(beta, os.w, rs.w)};
        float pw = from_west(p), pe = from_east(p);
        if (g.cx == 0) pw = fmaf(beta, e.w1, e.w0);
        if (g.cx == ROWT - 1) pe = fmaf(beta, e.e1, e.e0);
        const V4<float> ks = st_body(st, 2, row), kw = st_body(st, 3, row);
        V4<float> kn, ke;
        if (a.asym) {
          kn = ld4(Y.an32 + g.d0);
          ke = ld4(Y.ae32 + g.d0);
        } else {
          kn = st_north(st, 2, row, e.h2);
          float kwe = from_east(kw);
          if (g.cx == ROWT - 1) kwe = e.e2;
          ke = {kw.y, kw.z, kw.w, kwe};
        }
        V4<float> ap;
        ap.x = p.x + ks.x * ps.x + kn.x * pn.x + kw.x * pw + ke.x * p.y;
        ap.y = p.y + ks.y * ps.y + kn.y * pn.y + kw.y * p.x + ke.y * p.z;
        ap.z = p.z + ks.z * ps.z + kn.z * pn.z + kw.z * p.y + ke.z * p.w;
        ap.w = p.w + ks.w * ps.w + kn.w * pn.w + kw.w * p.z + ke.w * pe;
        if (!valid) return;
        if (a.dox) st4(Y.x32 + g.d0, x_plus_alpha_p(ld4(Y.x32 + g.d0), a.alpha, o0));
        st4(a.pnew + g.d0, p);
        st4(Y.ap32 + g.d0, ap);
        v[0] = double(ap.x) * double(p.x) + double(ap.y) * double(p.y) +
               double(ap.z) * double(p.z) + double(ap.w) * double(p.w);
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0) cg_matvec_epi(ctl[m], sum[0]);
      }));
}

template <bool FOLD>
__global__ void __launch_bounds__(NT, 3) k_mx_update_poly_st(DevStatic S, DevSystem Y,
                                                            Ctl *ctl, double *part, RedArgs ra) {
  struct A {
    bool skip;
    float alpha;
    float *rnew;
    const float *b[4];
  };
  quad_sweep_staged<2, 4, POLY_STAGES>(
      S, part, Y.err,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        const bool poly = Y.mpoly[m] && !unsym<true>(k);
        return A{(k.done | k.idone) != 0 || !poly, float(k.alpha), par ? Y.r32 : Y.r32b,
                 {par ? Y.r32b : Y.r32, Y.ap32, Y.as32, Y.aw32}};
      },
      [&](const A &a, const RowGeo &g, const StageRow &row) {
        Halo h{};
        if (row.north) {
          h.h0 = ld4(a.b[0] + g.dn);
          h.h1 = ld4(Y.ap32 + g.dn);
          h.h2 = ld4(Y.as32 + g.dn);
        } else if (row.south) {
          h.h0 = ld4(a.b[0] + g.ds);
          h.h1 = ld4(Y.ap32 + g.ds);
        }
        if (g.cx == 0) {
          h.w0 = a.b[0][g.dwe];
          h.w1 = Y.ap32[g.dwe];
        }
        if (g.cx == ROWT - 1) {
          h.e0 = a.b[0][g.dee];
          h.e1 = Y.ap32[g.dee];
          h.e2 = Y.aw32[g.dee];
        }
        return h;
      },
      [&](const A &a, const PolyStage &st, const StageRow &row, const RowGeo &g, bool valid,
          const Halo &e, double *v) {
        const float alpha = a.alpha;
        const V4<float> r0 = st_body(st, 0, row), a0 = st_body(st, 1, row);
        const V4<float> rn0 = {fmaf(-alpha, a0.x, r0.x), fmaf(-alpha, a0.y, r0.y),
                               fmaf(-alpha, a0.z, r0.z), fmaf(-alpha, a0.w, r0.w)};
        const V4<float> rN = st_north(st, 0, row, e.h0), aN = st_north(st, 1, row, e.h1);
        const V4<float> rS = st_south(st, 0, row, e.h0), aS = st_south(st, 1, row, e.h1);
        const V4<float> nN = {fmaf(-alpha, aN.x, rN.x), fmaf(-alpha, aN.y, rN.y),
                              fmaf(-alpha, aN.z, rN.z), fmaf(-alpha, aN.w, rN.w)};
        const V4<float> nS = {fmaf(-alpha, aS.x, rS.x), fmaf(-alpha, aS.y, rS.y),
                              fmaf(-alpha, aS.z, rS.z), fmaf(-alpha, aS.w, rS.w)};
        float nw = from_west(rn0), ne = from_east(rn0);
        if (g.cx == 0) nw = fmaf(-alpha, e.w1, e.w0);
        if (g.cx == ROWT - 1) ne = fmaf(-alpha, e.e1, e.e0);
        const V4<float> ks = st_body(st, 2, row), kw = st_body(st, 3, row);
        const V4<float> kn = st_north(st, 2, row, e.h2);
        float kwe = from_east(kw);
        if (g.cx == ROWT - 1) kwe = e.e2;
        const V4<float> ke = {kw.y, kw.z, kw.w, kwe};
        V4<float> zv;
        zv.x = rn0.x - (ks.x * nS.x + kn.x * nN.x + kw.x * nw + ke.x * rn0.y);
        zv.y = rn0.y - (ks.y * nS.y + kn.y * nN.y + kw.y * rn0.x + ke.y * rn0.z);
        zv.z = rn0.z - (ks.z * nS.z + kn.z * nN.z + kw.z * rn0.y + ke.z * rn0.w);
        zv.w = rn0.w - (ks.w * nS.w + kn.w * nN.w + kw.w * rn0.z + ke.w * ne);
        if (!valid) return;
        st4(a.rnew + g.d0, rn0);
        st4(Y.z32 + g.d0, zv);
        v[0] = double(rn0.x) * double(zv.x) + double(rn0.y) * double(zv.y) +
               double(rn0.z) * double(zv.z) + double(rn0.w) * double(zv.w);
        v[1] = double(rn0.x) * double(rn0.x) + double(rn0.y) * double(rn0.y) +
               double(rn0.z) * double(rn0.z) + double(rn0.w) * double(rn0.w);
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0)
          mx_update_epi(ctl[m], ra.glob, S.sc[m].iterm, sum[0], sum[1], 2.0, ra.no_stop);
      }));
}

template <bool FOLD>
__global__ void __launch_bounds__(NT, 4) k_mx_update_jac_st(DevStatic S, DevSystem Y,
                                                           Ctl *ctl, double *part, RedArgs ra) {
  struct A {
    bool skip;
    float alpha;
    float *rnew;
    const float *b[2];
  };
  quad_sweep_staged<2, 2, JAC_STAGES>(
      S, part, Y.err,
      [&](int m) {
        const Ctl &k = ctl[m];
        const bool par = k.parity;
        const bool poly = Y.mpoly[m] && !unsym<true>(k);
        return A{(k.done | k.idone) != 0 || poly, float(k.alpha), par ? Y.r32 : Y.r32b,
                 {par ? Y.r32b : Y.r32, Y.ap32}};
      },
      [&](const A &, const RowGeo &, const StageRow &) { return 0; },
      [&](const A &a, const JacStage &st, const StageRow &row, const RowGeo &g, bool valid,
          int, double *v) {
        if (!valid) return;
        const float alpha = a.alpha;
        V4<float> rv = st_body(st, 0, row);
        const V4<float> av = st_body(st, 1, row);
        rv.x = fmaf(-alpha, av.x, rv.x);
        rv.y = fmaf(-alpha, av.y, rv.y);
        rv.z = fmaf(-alpha, av.z, rv.z);
        rv.w = fmaf(-alpha, av.w, rv.w);
        st4(a.rnew + g.d0, rv);
        const double rr = double(rv.x) * double(rv.x) + double(rv.y) * double(rv.y) +
                          double(rv.z) * double(rv.z) + double(rv.w) * double(rv.w);
        v[0] = rr;
        v[1] = rr;
      },
      fold_if<FOLD>(ctl, [&](int m, const double *sum) {
        if (threadIdx.x == 0)
          mx_update_epi(ctl[m], ra.glob, S.sc[m].iterm, sum[0], sum[1], 2.0, ra.no_stop);
      }));
}

// Dynamic shared memory of a staged kernel (its stages), allowed once.
template <class K>
static size_t staged_smem(K kernel, size_t stage_bytes, int stages) {
  static std::mutex mu;
  static std::map<const void *, bool> done;
  const size_t bytes = size_t(stages) * stage_bytes;
  std::lock_guard<std::mutex> lock(mu);
  const void *k = reinterpret_cast<const void *>(kernel);
  if (!done[k]) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    done[k] = true;
  }
  return bytes;
}
template <class K>
static int staged_grid(const Launch &l, const DevStatic &S, K kernel, size_t smem, int cap) {
  static std::mutex mu;
  static std::map<const void *, int> cache;
  int b = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    const void *k = reinterpret_cast<const void *>(kernel);
    const auto it = cache.find(k);
    if (it != cache.end()) {
      b = it->second;
    } else {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, NT, smem);
      b = b > 0 ? b : 1;
      cache[k] = b;
    }
  }
  if (cap > 0) b = std::min(b, cap);
  return std::max(1, std::min(S.nquad, l.nsm * b));
}

static int reduce_grid(const DevStatic &S) { return std::min(S.nmember, 1024); }

// Resident CTAs per SM of a kernel (cached per kernel), for the grids of the
// kernel variants.
static int per_sm(const void *kernel) {
  static std::mutex mu;
  static std::map<const void *, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int a = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, kernel, NT, 0);
  a = a > 0 ? a : 1;
  cache[kernel] = a;
  return a;
}
// The grid of a quad kernel: its resident CTAs per SM (at most `cap` when
// cap > 0) times the SMs, at most one CTA per quad.
template <class K>
static int grid_of(const Launch &l, const DevStatic &S, K kernel, int cap) {
  int b = per_sm(reinterpret_cast<const void *>(kernel));
  if (cap > 0) b = std::min(b, cap);
  return std::max(1, std::min(S.nquad, l.nsm * b));
}

template <bool F>
static void mx_matvec_kernel(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                             double *part) {
  if (l.variant == 2) {
    if (l.may_asym) {
      const size_t sm = staged_smem(k_mx_matvec_st<true, F>, sizeof(MvStage), MV_STAGES);
      k_mx_matvec_st<true, F><<<staged_grid(l, S, k_mx_matvec_st<true, F>, sm, l.ctas_mv), NT,
                                sm, l.stream>>>(S, Y, ctl, part);
    } else {
      const size_t sm = staged_smem(k_mx_matvec_st<false, F>, sizeof(MvStage), MV_STAGES);
      k_mx_matvec_st<false, F><<<staged_grid(l, S, k_mx_matvec_st<false, F>, sm, l.ctas_mv), NT,
                                 sm, l.stream>>>(S, Y, ctl, part);
    }
  } else if (l.variant == 1) {
    if (l.may_asym)
      k_mx_matvec<true, 1, F><<<grid_of(l, S, k_mx_matvec<true, 1, F>, l.ctas_mv), NT, 0,
                                l.stream>>>(S, Y, ctl, part);
    else
      k_mx_matvec<false, 1, F><<<grid_of(l, S, k_mx_matvec<false, 1, F>, l.ctas_mv), NT, 0,
                                 l.stream>>>(S, Y, ctl, part);
  } else if (l.variant == 3) {
    if (l.may_asym)
      k_mx_matvec<true, 3, F><<<grid_of(l, S, k_mx_matvec<true, 3, F>, l.ctas_mv), NT, 0,
                                l.stream>>>(S, Y, ctl, part);
    else
      k_mx_matvec<false, 3, F><<<grid_of(l, S, k_mx_matvec<false, 3, F>, l.ctas_mv), NT, 0,
                                 l.stream>>>(S, Y, ctl, part);
  } else if (l.may_asym) {
    k_mx_matvec<true, 0, F><<<l.grid_cg32, NT, 0, l.stream>>>(S, Y, ctl, part);
  } else {
    k_mx_matvec<false, 0, F><<<l.grid_cg32, NT, 0, l.stream>>>(S, Y, ctl, part);
  }
  count_launches(1);
}
void launch_mx_matvec(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      double *part) {
  if (l.fold) {
    mx_matvec_kernel<true>(l, S, Y, ctl, part);
    return;
  }
  mx_matvec_kernel<false>(l, S, Y, ctl, part);
  launch_chan_mvmx(l, S, Y, ctl, part);
  k_red_mx_matvec<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, part);
  count_launches(1);
}
template <bool F>
static void mx_update_kernels(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                              double *part, const RedArgs &ra) {
  if (l.mx_jac && l.variant == 2) {
    const size_t sm = staged_smem(k_mx_update_jac_st<F>, sizeof(JacStage), JAC_STAGES);
    k_mx_update_jac_st<F><<<staged_grid(l, S, k_mx_update_jac_st<F>, sm, l.ctas_up), NT, sm,
                            l.stream>>>(S, Y, ctl, part, ra);
    count_launches(1);
  } else if (l.mx_jac) {
    if (l.variant == 1 || l.variant == 3)  // the Jacobi row already loads first
      k_mx_update_jac<1, F><<<grid_of(l, S, k_mx_update_jac<1, F>, l.ctas_up), NT, 0,
                              l.stream>>>(S, Y, ctl, part, ra);
    else
      k_mx_update_jac<0, F><<<l.grid_up32, NT, 0, l.stream>>>(S, Y, ctl, part, ra);
    count_launches(1);
  }
  if (l.mx_poly && l.variant == 2) {
    const size_t sm = staged_smem(k_mx_update_poly_st<F>, sizeof(PolyStage), POLY_STAGES);
    k_mx_update_poly_st<F><<<staged_grid(l, S, k_mx_update_poly_st<F>, sm, l.ctas_up), NT, sm,
                             l.stream>>>(S, Y, ctl, part, ra);
    count_launches(1);
  } else if (l.mx_poly) {
    if (l.variant == 1)
      k_mx_update_poly<1, F><<<grid_of(l, S, k_mx_update_poly<1, F>, l.ctas_up), NT, 0,
                               l.stream>>>(S, Y, ctl, part, ra);
    else if (l.variant == 3)
      k_mx_update_poly<3, F><<<grid_of(l, S, k_mx_update_poly<3, F>, l.ctas_up), NT, 0,
                               l.stream>>>(S, Y, ctl, part, ra);
    else
      k_mx_update_poly<0, F><<<l.grid_up32, NT, 0, l.stream>>>(S, Y, ctl, part, ra);
    count_launches(1);
  }
}
void launch_mx_update(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                      Glob *glob, double *part, int no_stop) {
  RedArgs ra{};
  ra.glob = glob;
  ra.no_stop = no_stop;
  if (l.fold) {
    mx_update_kernels<true>(l, S, Y, ctl, part, ra);
    return;
  }
  mx_update_kernels<false>(l, S, Y, ctl, part, ra);
  k_red_mx_update<<<reduce_grid(S), NT, 0, l.stream>>>(S, ctl, glob, part, 2.0, no_stop);
  count_launches(1);
}
void launch_mx_zinit(const Launch &l, const DevStatic &S, const DevSystem &Y, Ctl *ctl,
                     double *part) {
  if (!l.mx_poly) return;
  if (l.fold) {
    if (l.variant == 3)
      k_mx_zinit<true, true><<<grid_of(l, S, k_mx_zinit<true, true>, 0), NT, 0, l.stream>>>(
          S, Y, ctl, part);
    else
      k_mx_zinit<false, true><<<l.grid_up32, NT, 0, l.stream>>>(S, Y, ctl, part);
    count_launches(1);
    return;
  }
  if (l.variant == 3)
    k_mx_zinit<true, false><<<grid_of(l, S, k_mx_zinit<true, false>, 0), NT, 0, l.stream>>>(
        S, Y, ctl, part);
  else
    k_mx_zinit<false, false><<<l.grid_up32, NT, 0, l.stream>>>(S, Y, ctl, part);
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
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_mx_update_poly<0, false>, NT, 0);
  return b > 0 ? b : 1;
}

int occupancy_blocks_per_sm_mixed() {
  int a = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_mx_matvec<true, 0, false>, NT, 0);
  return a > 0 ? a : 1;
}

}  // namespace xm
