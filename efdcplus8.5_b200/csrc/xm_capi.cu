// xm_capi.cu -- the C-ABI of libefdc_xm (include/efdc_xm.h): context set-up
// (tile layout, device arrays), host<->device transfers, and the host-side
// orchestration of one CALPUV2C step (calpuv2c.f90:128-1187) and of CONGRAD.

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "xm_kernels.h"

namespace {

thread_local std::string g_last_error;

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

#define CK(expr)                                                                   \
  do {                                                                             \
    cudaError_t e__ = (expr);                                                      \
    if (e__ != cudaSuccess) {                                                      \
      set_error("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(e__)); \
      return EFDC_XM_CUDA_ERROR;                                                   \
    }                                                                              \
  } while (0)

std::atomic<long long> g_launches{0};

using xm::CopyJob;
using xm::Ctl;
using xm::TILE;

uint64_t morton2(uint32_t x, uint32_t y) {
  auto spread = [](uint64_t v) {
    v &= 0xffffffffull;
    v = (v | (v << 16)) & 0x0000ffff0000ffffull;
    v = (v | (v << 8)) & 0x00ff00ff00ff00ffull;
    v = (v | (v << 4)) & 0x0f0f0f0f0f0f0f0full;
    v = (v | (v << 2)) & 0x3333333333333333ull;
    v = (v | (v << 1)) & 0x5555555555555555ull;
    return v;
  };
  return spread(x) | (spread(y) << 1);
}

}  // namespace

namespace xm {
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void set_last_error_str(const char *msg) { g_last_error = msg ? msg : ""; }
}  // namespace xm

// A device buffer owned by the context.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

struct efdc_xm_ctx {
  int device = 0;
  int la = 0, lc = 0;
  int ntile = 0, nslot = 0, grid = 1, grid_cg = 1, grid_mv64 = 1, grid_cg32 = 1, grid_up32 = 1, nsm = 0;
  cudaStream_t stream = nullptr;
  std::vector<DevBuf> bufs;
  // host copies of the layout
  std::vector<int> slot_of_L;  // [lc+1], slot of water cell L (0 otherwise)
  std::vector<int> lidx_h;     // [nslot]
  // device views
  xm::DevStatic S{};
  xm::DevState X{};
  xm::DevSystem Y{};
  xm::DevObc B{};
  Ctl *ctl = nullptr;
  Ctl *ctl_h = nullptr;  // pinned mirror
  double *part = nullptr;
  int *lidx = nullptr;
  // staging: device buffers in host (L) order, one per transferable array
  std::vector<double *> stage;
  CopyJob *jobs_d = nullptr;
  CopyJob *jobs_h = nullptr;  // pinned
  int max_jobs = 0;
  // open boundaries
  bool obc_serial = false;
  bool may_asym = false;  // a radiation boundary exists: the operator can be unsymmetric
  int nobc = 0;
  int side_n[4] = {0, 0, 0, 0};
  std::vector<double> tcp;
  int mtide = 0;
  double *pser_d = nullptr;
  double *pser_h = nullptr;  // pinned
  double *ptmp = nullptr;    // scratch P for kernel timing
  // bookkeeping
  int last_iters = 8;
  int last_inner = 8;
  int last_n = 0, last_ntstbc = 0, last_isdry = 0;
  std::vector<int32_t> oldmask_h;

  template <class T>
  T *alloc(size_t n, bool zero = true) {
    DevBuf b;
    b.bytes = std::max<size_t>(n, 1) * sizeof(T);
    if (cudaMalloc(&b.p, b.bytes) != cudaSuccess) return nullptr;
    if (zero) cudaMemset(b.p, 0, b.bytes);
    bufs.push_back(b);
    return static_cast<T *>(b.p);
  }
  xm::Launch L() const { return xm::Launch{grid, grid_cg, grid_mv64, grid_cg32, grid_up32, ntile, stream}; }
};

namespace {

// Scatter host-order device staging buffers into tile-order arrays.
int run_scatter(efdc_xm_ctx *c, const std::vector<CopyJob> &jobs) {
  if (jobs.empty()) return EFDC_XM_OK;
  for (size_t base = 0; base < jobs.size(); base += c->max_jobs) {
    const int n = int(std::min<size_t>(c->max_jobs, jobs.size() - base));
    std::memcpy(c->jobs_h, jobs.data() + base, n * sizeof(CopyJob));
    CK(cudaMemcpyAsync(c->jobs_d, c->jobs_h, n * sizeof(CopyJob), cudaMemcpyHostToDevice, c->stream));
    xm::launch_scatter(c->stream, c->jobs_d, n, c->lidx, c->nslot, c->lc);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
  }
  return EFDC_XM_OK;
}

int run_gather(efdc_xm_ctx *c, const std::vector<CopyJob> &jobs) {
  if (jobs.empty()) return EFDC_XM_OK;
  for (size_t base = 0; base < jobs.size(); base += c->max_jobs) {
    const int n = int(std::min<size_t>(c->max_jobs, jobs.size() - base));
    std::memcpy(c->jobs_h, jobs.data() + base, n * sizeof(CopyJob));
    CK(cudaMemcpyAsync(c->jobs_d, c->jobs_h, n * sizeof(CopyJob), cudaMemcpyHostToDevice, c->stream));
    xm::launch_gather(c->stream, c->jobs_d, n, c->lidx, c->nslot);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
  }
  return EFDC_XM_OK;
}

// Transfer plan entry: a host array (element L at [L-1], LC elements) and the
// tile-order device array it maps to.
struct Xfer {
  const void *host;
  void *dev;
  int kind;  // 0 double, 1 LOGICAL (normalised to 0/1), 2 raw int, 3 double water-only
};

int upload_arrays(efdc_xm_ctx *c, const std::vector<Xfer> &xs) {
  std::vector<CopyJob> jobs;
  size_t k = 0;
  for (const Xfer &x : xs) {
    if (!x.host || !x.dev) continue;
    if (k >= c->stage.size()) {
      set_error("internal: staging exhausted");
      return EFDC_XM_CUDA_ERROR;
    }
    const size_t bytes = size_t(c->lc) * ((x.kind == 1 || x.kind == 2) ? sizeof(int32_t) : sizeof(double));
    CK(cudaMemcpyAsync(c->stage[k], x.host, bytes, cudaMemcpyHostToDevice, c->stream));
    jobs.push_back(CopyJob{c->stage[k], x.dev, x.kind});
    ++k;
  }
  return run_scatter(c, jobs);
}

int download_arrays(efdc_xm_ctx *c, const std::vector<Xfer> &xs) {
  std::vector<CopyJob> jobs;
  std::vector<std::pair<void *, size_t>> dst;
  size_t k = 0;
  for (const Xfer &x : xs) {
    if (!x.host || !x.dev) continue;
    // the gather fills elements L=2..LA (indices 1..LA-1); only that range
    // goes back, so the caller's ghost elements 1 and LC are left alone
    const size_t esz = ((x.kind == 1 || x.kind == 2) ? sizeof(int32_t) : sizeof(double));
    jobs.push_back(CopyJob{c->stage[k], x.dev, x.kind});
    dst.push_back({const_cast<void *>(x.host), esz});
    ++k;
  }
  int rc = run_gather(c, jobs);
  if (rc) return rc;
  for (size_t i = 0; i < dst.size(); ++i) {
    const size_t esz = dst[i].second;
    CK(cudaMemcpyAsync(static_cast<char *>(dst[i].first) + esz,
                       reinterpret_cast<const char *>(c->stage[i]) + esz, esz * size_t(c->la - 1),
                       cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return EFDC_XM_OK;
}

int read_ctl(efdc_xm_ctx *c) {
  CK(cudaMemcpyAsync(c->ctl_h, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EFDC_XM_OK;
}

int write_ctl(efdc_xm_ctx *c) {
  CK(cudaMemcpyAsync(c->ctl, c->ctl_h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
  return EFDC_XM_OK;
}

// FP64 CONGRAD on the scaled system in c->Y, P = c->X.p (or `P`).
int solve_fp64(efdc_xm_ctx *c, double *P, double rsqm, int iterm, int *iters, double *rsq,
               int *status) {
  const xm::Launch l = c->L();
  xm::launch_cg_init(l, c->S, c->Y, P, c->ctl, c->part);
  CK(cudaGetLastError());
  int launched = 0;
  int chunk = std::max(1, std::min(c->last_iters, iterm));
  for (;;) {
    for (int k = 0; k < chunk && launched < iterm; ++k, ++launched)
      xm::launch_cg_iter(l, c->S, c->Y, P, c->ctl, c->part, rsqm, iterm);
    CK(cudaGetLastError());
    int rc = read_ctl(c);
    if (rc) return rc;
    if (c->ctl_h->done || launched >= iterm) break;
    chunk = 4;
  }
  *iters = c->ctl_h->iter;
  *rsq = c->ctl_h->rsq;
  *status = c->ctl_h->status;
  if (!c->ctl_h->done) *status = EFDC_XM_CG_MAXITER;
  if (*iters > 0) c->last_iters = *iters;
  return EFDC_XM_OK;
}

// MIXED: FP64 refinement around the FP32 inner PCG.
int solve_mixed(efdc_xm_ctx *c, double *P, double rsqm_ref, int iterm, int *iters, double *rsq,
                int *status, int *outer, double factor) {
  const xm::Launch l = c->L();
  // the FP32 path stops on the FP64 residual, past the reference's RSQM
  const double rsqm = rsqm_ref * (factor > 0 ? factor : 0.1);
  const int total_cap = 2 * iterm + 50;
  const int max_outer = 30;
  const double rel_tol = 1e-6;  // inner: |r| down 1e-6 (FP32 reaches ~1e-7 here)
  // reset the solve bookkeeping
  int rc = read_ctl(c);
  if (rc) return rc;
  c->ctl_h->iter = 0;
  c->ctl_h->outer = 0;
  c->ctl_h->done = 0;
  c->ctl_h->idone = 0;
  c->ctl_h->status = 0;
  c->ctl_h->counter = 0;
  rc = write_ctl(c);
  if (rc) return rc;
  bool converged = false;
  for (int o = 0; o < max_outer; ++o) {
    xm::launch_mx_resid(l, c->S, c->Y, P, c->ctl, c->part, rsqm, rel_tol);
    CK(cudaGetLastError());
    rc = read_ctl(c);
    if (rc) return rc;
    if (c->ctl_h->done) {
      converged = (c->ctl_h->status == 0);
      break;
    }
    if (c->ctl_h->iter >= total_cap) break;
    int chunk = std::max(1, c->last_inner);
    for (;;) {
      for (int k = 0; k < chunk; ++k)
        xm::launch_mx_iter(l, c->S, c->Y, c->ctl, c->part, iterm, total_cap);
      CK(cudaGetLastError());
      rc = read_ctl(c);
      if (rc) return rc;
      if (c->ctl_h->idone || c->ctl_h->done) break;
      chunk = 4;
    }
    if (c->ctl_h->inner_iter > 0) c->last_inner = c->ctl_h->inner_iter;
    if (c->ctl_h->done) break;  // non-finite
    xm::launch_mx_apply(l, c->S, c->Y, P);
    CK(cudaGetLastError());
  }
  *iters = c->ctl_h->iter;
  *rsq = c->ctl_h->rsq64;
  *outer = c->ctl_h->outer;
  *status = c->ctl_h->status;
  if (*status == 0 && !converged) *status = EFDC_XM_CG_MAXITER;
  return EFDC_XM_OK;
}

xm::StepScalars make_scalars(const efdc_xm_ctx *c, const efdc_xm_params *p) {
  xm::StepScalars s{};
  s.delt = p->delt;
  s.deltd2 = 0.5 * p->delt;  // calpuv2c.f90:129-135
  s.delti = 1. / p->delt;
  s.g = p->g;
  s.gi = 1. / p->g;  // aaefdc.f90:648
  s.hdry = p->hdry;
  s.rsqm = p->rsqm;
  s.snlt = p->snlt;
  s.ritb1 = p->ritb1;
  s.isdry = p->isdry;
  s.ndrystp = p->ndrystp;
  s.isbal = p->isbal;
  s.iterm = p->iterm;
  // setopenbc.f90:24-29 on the host, libm as the reference
  for (int m = 0; m < c->mtide && m < xm::MT_MAX; ++m) {
    double TM = std::fmod(p->tn, c->tcp[m]);
    TM = p->pi2 * TM / c->tcp[m];
    s.cosv[m] = std::cos(TM);
    s.sinv[m] = std::sin(TM);
  }
  return s;
}

}  // namespace

extern "C" {

int32_t efdc_xm_abi_version(void) { return EFDC_XM_ABI_VERSION; }

const char *efdc_xm_last_error(void) { return g_last_error.c_str(); }

void efdc_xm_destroy(efdc_xm_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto &b : c->bufs) cudaFree(b.p);
  if (c->ctl_h) cudaFreeHost(c->ctl_h);
  if (c->jobs_h) cudaFreeHost(c->jobs_h);
  if (c->pser_h) cudaFreeHost(c->pser_h);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

efdc_xm_ctx *efdc_xm_create(const efdc_xm_grid *g, int32_t device) {
  g_last_error.clear();
  if (!g) {
    set_error("efdc_xm_create: grid is NULL");
    return nullptr;
  }
  const int la = g->la, lc = g->lc;
  if (la < 2 || lc != la + 1) {
    set_error("efdc_xm_create: need LA >= 2 and LC == LA+1 (got LA=%d LC=%d)", la, lc);
    return nullptr;
  }
  if (!g->il || !g->jl || !g->lnc || !g->lsc || !g->lec || !g->lwc) {
    set_error("efdc_xm_create: IL, JL and the four neighbour maps are required");
    return nullptr;
  }
  const double *req[] = {g->dxyp, g->dxyip, g->dxiu, g->dyiu, g->dxiv, g->dyiv, g->dxyu, g->dxyv,
                         g->hruo, g->hrvo, g->subo, g->svbo, g->sbxo, g->sbyo, g->belv};
  for (const double *r : req)
    if (!r) {
      set_error("efdc_xm_create: a metric array is NULL");
      return nullptr;
    }
  if (g->mtide < 0 || g->mtide > xm::MT_MAX || (g->mtide > 0 && !g->tcp)) {
    set_error("efdc_xm_create: MTIDE must be in 0..%d with TCP given", xm::MT_MAX);
    return nullptr;
  }
  // ---- structured-grid check and tile layout (host) ----
  int imin = INT32_MAX, imax = INT32_MIN, jmin = INT32_MAX, jmax = INT32_MIN;
  for (int L = 2; L <= la; ++L) {
    imin = std::min(imin, g->il[L - 1]);
    imax = std::max(imax, g->il[L - 1]);
    jmin = std::min(jmin, g->jl[L - 1]);
    jmax = std::max(jmax, g->jl[L - 1]);
  }
  const long ni = long(imax) - imin + 1, nj = long(jmax) - jmin + 1;
  if (ni <= 0 || nj <= 0 || ni * nj > (1L << 31) - 1) {
    set_error("efdc_xm_create: bad IL/JL range");
    return nullptr;
  }
  std::vector<int> lij(size_t(ni * nj), 0);
  for (int L = 2; L <= la; ++L) {
    const long k = long(g->jl[L - 1] - jmin) * ni + (g->il[L - 1] - imin);
    if (lij[k]) {
      set_error("efdc_xm_create: cells %d and %d share (I,J)", lij[k], L);
      return nullptr;
    }
    lij[k] = L;
  }
  auto at = [&](long i, long j) -> int {
    if (i < imin || i > imax || j < jmin || j > jmax) return lc;
    const int L = lij[size_t(long(j - jmin) * ni + (i - imin))];
    return L ? L : lc;
  };
  for (int L = 2; L <= la; ++L) {
    const int i = g->il[L - 1], j = g->jl[L - 1];
    if (g->lec[L - 1] != at(i + 1, j) || g->lwc[L - 1] != at(i - 1, j) ||
        g->lnc[L - 1] != at(i, j + 1) || g->lsc[L - 1] != at(i, j - 1)) {
      set_error("efdc_xm_create: cell L=%d (I=%d,J=%d): LNC/LSC/LEC/LWC are not the maps of a "
                "structured grid (periodic ISCONNECT links are not supported)", L, i, j);
      return nullptr;
    }
  }
  const int ntx = int((ni + xm::TX - 1) / xm::TX), nty = int((nj + xm::TY - 1) / xm::TY);
  std::vector<int> tile_of(size_t(ntx) * nty, 0);
  std::vector<std::pair<uint64_t, int>> act;
  for (int L = 2; L <= la; ++L) {
    const int tx = (g->il[L - 1] - imin) / xm::TX, ty = (g->jl[L - 1] - jmin) / xm::TY;
    int &t = tile_of[size_t(ty) * ntx + tx];
    if (!t) {
      t = -1;
      act.push_back({morton2(tx, ty), ty * ntx + tx});
    }
  }
  std::sort(act.begin(), act.end());
  for (size_t k = 0; k < act.size(); ++k) tile_of[act[k].second] = int(k) + 1;

  efdc_xm_ctx *c = new efdc_xm_ctx();
  c->device = device;
  c->la = la;
  c->lc = lc;
  c->ntile = int(act.size()) + 1;
  c->nslot = c->ntile * TILE;
  auto bail = [&](const char *what) -> efdc_xm_ctx * {
    if (g_last_error.empty()) set_error("efdc_xm_create: %s", what);
    efdc_xm_destroy(c);
    return nullptr;
  };
  if (cudaSetDevice(device) != cudaSuccess) {
    set_error("efdc_xm_create: cudaSetDevice(%d) failed", device);
    delete c;
    return nullptr;
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail("stream creation failed");
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
  const int occ = xm::occupancy_blocks_per_sm();
  const int occ_cg = xm::occupancy_blocks_per_sm_cg();
  const int occ_cg32 = xm::occupancy_blocks_per_sm_mixed();
  c->grid = std::max(1, std::min(c->ntile - 1, c->nsm * occ));
  c->grid_cg = std::max(1, std::min((c->ntile - 1 + 3) / 4, c->nsm * occ_cg));
  c->grid_cg32 = std::max(1, std::min((c->ntile - 1 + 3) / 4, c->nsm * occ_cg32));
  c->grid_mv64 = std::max(1, std::min((c->ntile - 1 + 3) / 4, c->nsm * xm::occupancy_blocks_per_sm_mv64()));
  c->grid_up32 = std::max(1, std::min((c->ntile - 1 + 3) / 4, c->nsm * xm::occupancy_blocks_per_sm_mixed_update()));

  std::vector<int4> tnbr(c->ntile, int4{0, 0, 0, 0});
  std::vector<uint8_t> kind(c->nslot, xm::LAND);
  c->lidx_h.assign(c->nslot, 0);
  c->slot_of_L.assign(size_t(lc) + 1, 0);
  for (size_t k = 0; k < act.size(); ++k) {
    const int id = act[k].second, tx = id % ntx, ty = id / ntx;
    auto tl = [&](int x, int y) { return (x < 0 || y < 0 || x >= ntx || y >= nty) ? 0 : std::max(tile_of[size_t(y) * ntx + x], 0); };
    tnbr[k + 1] = int4{tl(tx - 1, ty), tl(tx + 1, ty), tl(tx, ty - 1), tl(tx, ty + 1)};
  }
  for (int L = 2; L <= la; ++L) {
    const int ii = g->il[L - 1] - imin, jj = g->jl[L - 1] - jmin;
    const int t = tile_of[size_t(jj / xm::TY) * ntx + ii / xm::TX];
    const int d = t * TILE + (jj % xm::TY) * xm::TX + (ii % xm::TX);
    kind[d] = xm::WATER;
    c->lidx_h[d] = L;
    c->slot_of_L[L] = d;
  }
  // ---- open boundaries ----
  std::vector<int> bslot, bnbr, bside, bispb;
  std::vector<double> bpcb, bpsb;
  c->mtide = g->mtide;
  c->tcp.assign(g->tcp, g->tcp + g->mtide);
  for (int s = 0; s < 4; ++s) {
    const efdc_xm_obc &o = g->obc[s];
    if (o.n < 0 || (o.n > 0 && (!o.l || !o.ispb))) return bail("bad open-boundary arrays");
    c->side_n[s] = o.n;
    for (int ll = 0; ll < o.n; ++ll) {
      const int L = o.l[ll];
      if (L < 2 || L > la) return bail("open-boundary L out of range");
      const int nbL = (s == 0) ? g->lec[L - 1] : (s == 1) ? g->lwc[L - 1] : (s == 2) ? g->lnc[L - 1] : g->lsc[L - 1];
      bslot.push_back(c->slot_of_L[L]);
      bnbr.push_back(nbL == lc ? 0 : c->slot_of_L[nbL]);  // 0 = a slot of the ghost tile
      bside.push_back(s);
      bispb.push_back(o.ispb[ll]);
      for (int m = 0; m < g->mtide; ++m) {
        bpcb.push_back(o.pcb ? o.pcb[size_t(m) * o.ld + ll] : 0.0);
        bpsb.push_back(o.psb ? o.psb[size_t(m) * o.ld + ll] : 0.0);
      }
      kind[c->slot_of_L[L]] = xm::OPENBC;
      if (o.ispb[ll] == 1 || o.ispb[ll] == 2) c->may_asym = true;
    }
  }
  c->nobc = int(bslot.size());
  {  // hazard check: unique interior targets that are not boundary cells
    std::unordered_map<int, int> seen;
    std::vector<char> isbc(c->nslot, 0);
    for (int d : bslot) isbc[d] = 1;
    bool serial = false;
    for (size_t k = 0; k < bslot.size(); ++k) {
      const int nb = bnbr[k];
      if (nb == 0 || isbc[nb] || seen.count(nb)) serial = true;
      seen[nb] = 1;
    }
    c->obc_serial = serial;
  }
  // ---- device arrays ----
  const size_t ns = c->nslot;
  c->lidx = c->alloc<int>(ns);
  int4 *tnbr_d = c->alloc<int4>(c->ntile);
  uint8_t *kind_d = c->alloc<uint8_t>(ns);
  if (!c->lidx || !tnbr_d || !kind_d) return bail("cudaMalloc failed");
  cudaMemcpy(c->lidx, c->lidx_h.data(), ns * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(tnbr_d, tnbr.data(), tnbr.size() * sizeof(int4), cudaMemcpyHostToDevice);
  cudaMemcpy(kind_d, kind.data(), ns, cudaMemcpyHostToDevice);
  auto D = [&]() { return c->alloc<double>(ns); };
  auto I = [&]() { return c->alloc<int>(ns); };
  auto Fl = [&]() { return c->alloc<float>(ns); };
  xm::DevStatic &S = c->S;
  S.tnbr = tnbr_d;
  S.kind = kind_d;
  S.lidx = c->lidx;
  double *st[18];
  for (double *&p : st) p = D();
  S.dxyp = st[0]; S.dxyip = st[1]; S.dxiu = st[2]; S.dyiu = st[3]; S.dxiv = st[4];
  S.dyiv = st[5]; S.dxyu = st[6]; S.dxyv = st[7]; S.hruo = st[8]; S.hrvo = st[9];
  S.subo = st[10]; S.svbo = st[11]; S.sbxo = st[12]; S.sbyo = st[13]; S.belv = st[14];
  S.rcx = st[15]; S.fsgzu = st[16]; S.fsgzv = st[17];
  xm::DevState &X = c->X;
  X.p = D(); X.hp = D(); X.h1p = D(); X.hu = D(); X.hv = D(); X.uhdye = D(); X.vhdxe = D();
  X.sub = D(); X.svb = D(); X.sbx = D(); X.sby = D();
  X.lmaskdry = I(); X.iscdry = I(); X.lopenbcdry = I(); X.natdry = I(); X.oldmask = I();
  double *fin[9];
  for (double *&p : fin) p = D();
  X.fcaxe = fin[0]; X.fcaye = fin[1]; X.fxe = fin[2]; X.fye = fin[3]; X.tsx = fin[4];
  X.tsy = fin[5]; X.tbx = fin[6]; X.tby = fin[7]; X.qsume = fin[8];
  X.uhe = D(); X.vhe = D(); X.hpi = D(); X.hui = D(); X.hvi = D(); X.qdwaste = D(); X.vdwaste = D();
  X.uhdy1e = D(); X.vhdx1e = D(); X.sub1 = D(); X.svb1 = D(); X.fp1 = D(); X.fuhdye = D();
  X.fvhdxe = D(); X.fp = D(); X.cc = D(); X.cs = D(); X.cw = D(); X.ce = D(); X.cn = D();
  X.wd_act = I(); X.sub_n = D(); X.svb_n = D(); X.sbx_n = D(); X.sby_n = D(); X.wasted = I();
  xm::DevSystem &Y = c->Y;
  Y.ccc = D(); Y.ccs = D(); Y.ccw = D(); Y.cce = D(); Y.ccn = D(); Y.fptmp = D();
  Y.r = D(); Y.pa = D(); Y.pb = D(); Y.ap = D();
  Y.as32 = Fl(); Y.aw32 = Fl(); Y.ae32 = Fl(); Y.an32 = Fl();
  Y.r32 = Fl(); Y.pa32 = Fl(); Y.pb32 = Fl(); Y.ap32 = Fl(); Y.x32 = Fl();
  c->ptmp = D();
  c->ctl = c->alloc<Ctl>(1);
  c->part = c->alloc<double>(size_t(2) * std::max(std::max(c->grid, c->grid_up32),
                                                  std::max(c->grid_cg, c->grid_cg32)) + 64);
  if (!Y.x32 || !c->ctl || !c->part) return bail("cudaMalloc failed (device memory)");
  if (cudaHostAlloc(reinterpret_cast<void **>(&c->ctl_h), sizeof(Ctl), cudaHostAllocDefault) != cudaSuccess)
    return bail("cudaHostAlloc failed");
  std::memset(c->ctl_h, 0, sizeof(Ctl));
  // land slots of the scaled system: CCC=1 keeps them inert in the CG
  {
    std::vector<double> one(ns, 0.0);
    for (size_t d = 0; d < ns; ++d)
      if (kind[d] == xm::LAND) one[d] = 1.0;
    cudaMemcpy(Y.ccc, one.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
    // RCX/RCY: 1 on water cells, 0 on the ghosts (calpuv2c.f90:97-102)
    std::vector<double> rc(ns, 0.0), fu(ns, 1.0), fv(ns, 1.0);
    for (int L = 2; L <= la; ++L) {
      const int d = c->slot_of_L[L];
      rc[d] = 1.0;
      fu[d] = 0.5 / g->dxyu[L - 1];  // calpuv2c.f90:111-116
      fv[d] = 0.5 / g->dxyv[L - 1];
    }
    cudaMemcpy(st[15], rc.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(st[16], fu.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(st[17], fv.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
  }
  // staging buffers (host order) and copy jobs
  const int nstage = 40;
  for (int k = 0; k < nstage; ++k) {
    double *p = c->alloc<double>(size_t(lc) + 1, false);
    if (!p) return bail("cudaMalloc failed (staging)");
    c->stage.push_back(p);
  }
  c->max_jobs = 64;
  c->jobs_d = c->alloc<CopyJob>(c->max_jobs);
  if (cudaHostAlloc(reinterpret_cast<void **>(&c->jobs_h), c->max_jobs * sizeof(CopyJob), cudaHostAllocDefault) != cudaSuccess)
    return bail("cudaHostAlloc failed");
  // open-boundary device arrays
  xm::DevObc &Bo = c->B;
  Bo.n = c->nobc;
  Bo.mtide = g->mtide;
  if (c->nobc > 0) {
    int *bs = c->alloc<int>(c->nobc), *bn = c->alloc<int>(c->nobc), *bd = c->alloc<int>(c->nobc),
        *bi = c->alloc<int>(c->nobc);
    double *pc = c->alloc<double>(std::max<size_t>(bpcb.size(), 1)),
           *ps = c->alloc<double>(std::max<size_t>(bpsb.size(), 1));
    c->pser_d = c->alloc<double>(c->nobc);
    if (!bs || !bn || !bd || !bi || !pc || !ps || !c->pser_d) return bail("cudaMalloc failed (obc)");
    cudaMemcpy(bs, bslot.data(), c->nobc * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(bn, bnbr.data(), c->nobc * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(bd, bside.data(), c->nobc * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(bi, bispb.data(), c->nobc * sizeof(int), cudaMemcpyHostToDevice);
    if (!bpcb.empty()) {
      cudaMemcpy(pc, bpcb.data(), bpcb.size() * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(ps, bpsb.data(), bpsb.size() * sizeof(double), cudaMemcpyHostToDevice);
    }
    Bo.slot = bs;
    Bo.nbr = bn;
    Bo.side = bd;
    Bo.ispb = bi;
    Bo.pcb = pc;
    Bo.psb = ps;
    Bo.pser = c->pser_d;
    if (cudaHostAlloc(reinterpret_cast<void **>(&c->pser_h), c->nobc * sizeof(double), cudaHostAllocDefault) != cudaSuccess)
      return bail("cudaHostAlloc failed");
  }
  // the zero-fills above ran on the legacy stream; finish them before any
  // work on the non-blocking solver stream
  if (cudaDeviceSynchronize() != cudaSuccess) return bail("device error during allocation");
  // static metrics into tile order (land slots take element LC)
  std::vector<Xfer> xs = {
      {g->dxyp, st[0], 0}, {g->dxyip, st[1], 0}, {g->dxiu, st[2], 0}, {g->dyiu, st[3], 0},
      {g->dxiv, st[4], 0}, {g->dyiv, st[5], 0}, {g->dxyu, st[6], 0}, {g->dxyv, st[7], 0},
      {g->hruo, st[8], 0}, {g->hrvo, st[9], 0}, {g->subo, st[10], 0}, {g->svbo, st[11], 0},
      {g->sbxo, st[12], 0}, {g->sbyo, st[13], 0}, {g->belv, st[14], 0}};
  if (upload_arrays(c, xs) != EFDC_XM_OK) return bail("upload of the static arrays failed");
  if (cudaDeviceSynchronize() != cudaSuccess) return bail("device error during set-up");
  return c;
}

int32_t efdc_xm_upload(efdc_xm_ctx *c, const efdc_xm_fields *f) {
  if (!c || !f) {
    set_error("efdc_xm_upload: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  xm::DevState &X = c->X;
  std::vector<Xfer> xs = {
      {f->p, X.p, 0}, {f->hp, X.hp, 0}, {f->hu, X.hu, 0}, {f->hv, X.hv, 0},
      {f->uhdye, X.uhdye, 0}, {f->vhdxe, X.vhdxe, 0}, {f->sub, X.sub, 0}, {f->svb, X.svb, 0},
      {f->sbx, X.sbx, 0}, {f->sby, X.sby, 0}, {f->lmaskdry, X.lmaskdry, 1},
      {f->iscdry, X.iscdry, 2}, {f->lopenbcdry, X.lopenbcdry, 1}, {f->natdry, X.natdry, 2},
      {f->fcaxe, const_cast<double *>(X.fcaxe), 0}, {f->fcaye, const_cast<double *>(X.fcaye), 0},
      {f->fxe, const_cast<double *>(X.fxe), 0}, {f->fye, const_cast<double *>(X.fye), 0},
      {f->tsx, const_cast<double *>(X.tsx), 0}, {f->tsy, const_cast<double *>(X.tsy), 0},
      {f->tbx, const_cast<double *>(X.tbx), 0}, {f->tby, const_cast<double *>(X.tby), 0},
      {f->qsume, const_cast<double *>(X.qsume), 0}, {f->qdwaste, X.qdwaste, 0},
      {f->vdwaste, X.vdwaste, 0}};
  int rc = upload_arrays(c, xs);
  if (rc) return rc;
  // the second buffer of each time-level pair starts as a copy (its land
  // slots must hold the ghost values too); the H1P input is not used because
  // a step begins with H1P = HP (calpuv2c.f90:264)
  const size_t nb = size_t(c->nslot) * sizeof(double);
  if (f->uhdye) CK(cudaMemcpyAsync(X.uhdy1e, X.uhdye, nb, cudaMemcpyDeviceToDevice, c->stream));
  if (f->vhdxe) CK(cudaMemcpyAsync(X.vhdx1e, X.vhdxe, nb, cudaMemcpyDeviceToDevice, c->stream));
  if (f->hp) CK(cudaMemcpyAsync(X.h1p, X.hp, nb, cudaMemcpyDeviceToDevice, c->stream));
  if (c->nobc > 0) {
    int k = 0;
    for (int s = 0; s < 4; ++s)
      for (int ll = 0; ll < c->side_n[s]; ++ll, ++k) c->pser_h[k] = f->pser[s] ? f->pser[s][ll] : 0.0;
    CK(cudaMemcpyAsync(c->pser_d, c->pser_h, c->nobc * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  if (f->lmaskdry) c->oldmask_h.assign(f->lmaskdry, f->lmaskdry + c->lc);
  return EFDC_XM_OK;
}

int32_t efdc_xm_download(efdc_xm_ctx *c, efdc_xm_fields *f) {
  if (!c || !f) {
    set_error("efdc_xm_download: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  xm::DevState &X = c->X;
  std::vector<int32_t> oldmask;
  const bool lists = f->lwet || f->ldry;
  if (lists) oldmask.assign(c->lc, 1);
  std::vector<Xfer> xs = {
      {f->p, X.p, 0}, {f->hp, X.hp, 0}, {f->h1p, X.h1p, 0}, {f->hu, X.hu, 0}, {f->hv, X.hv, 0},
      {f->uhdye, X.uhdye, 0}, {f->vhdxe, X.vhdxe, 0}, {f->sub, X.sub, 0}, {f->svb, X.svb, 0},
      {f->sbx, X.sbx, 0}, {f->sby, X.sby, 0}, {f->lmaskdry, X.lmaskdry, 1},
      {f->iscdry, X.iscdry, 2}, {f->lopenbcdry, X.lopenbcdry, 1}, {f->natdry, X.natdry, 2},
      {f->uhe, X.uhe, 0}, {f->vhe, X.vhe, 0}, {f->hpi, X.hpi, 0}, {f->hui, X.hui, 0},
      {f->hvi, X.hvi, 0}, {f->qdwaste, X.qdwaste, 0}, {f->vdwaste, X.vdwaste, 0},
      {f->ccc, c->Y.ccc, 0}, {f->ccs, c->Y.ccs, 0}, {f->ccw, c->Y.ccw, 0}, {f->cce, c->Y.cce, 0},
      {f->ccn, c->Y.ccn, 0}, {f->fptmp, c->Y.fptmp, 0},
      {lists ? oldmask.data() : nullptr, X.oldmask, 2}};
  int rc = download_arrays(c, xs);
  if (rc) return rc;
  if (lists) {  // calpuv2c.f90:1061-1080 (L order)
    std::vector<int32_t> mask(c->lc, 1);
    if (c->last_isdry > 0) {
      std::vector<Xfer> m = {{mask.data(), X.lmaskdry, 1}};
      if ((rc = download_arrays(c, m))) return rc;
    }
    int nw = 0, nd = 0;
    for (int L = 2; L <= c->la; ++L) {
      if (c->last_isdry == 0 || mask[L - 1]) {
        if (f->lwet) f->lwet[nw] = L;
        ++nw;
      } else if (oldmask[L - 1] || c->last_n < c->last_ntstbc + 1) {
        if (f->ldry) f->ldry[nd] = L;
        ++nd;
      }
    }
  }
  return EFDC_XM_OK;
}

int32_t efdc_xm_step_device(efdc_xm_ctx *c, const efdc_xm_params *prm, efdc_xm_stats *stats) {
  efdc_xm_stats dummy;
  if (!stats) stats = &dummy;
  std::memset(stats, 0, sizeof(*stats));
  if (!c || !prm) {
    set_error("efdc_xm_step_device: NULL argument");
    return stats->status = EFDC_XM_BAD_ARGUMENT;
  }
  if (!(prm->delt > 0) || prm->iterm < 1 || prm->g <= 0) {
    set_error("efdc_xm_step_device: need DELT > 0, G > 0, ITERM >= 1");
    return stats->status = EFDC_XM_BAD_ARGUMENT;
  }
  if (prm->precision != EFDC_XM_PREC_FP64 && prm->precision != EFDC_XM_PREC_MIXED) {
    set_error("efdc_xm_step_device: unknown precision %d", prm->precision);
    return stats->status = EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  const xm::StepScalars s = make_scalars(c, prm);
  const xm::Launch l = c->L();
  const bool mixed = prm->precision == EFDC_XM_PREC_MIXED;
  const int max_sweeps = prm->max_sweeps > 0 ? prm->max_sweeps : 500;
  c->last_n = prm->n;
  c->last_ntstbc = prm->ntstbc;
  c->last_isdry = prm->isdry;

  // counters of this step
  int rc = read_ctl(c);
  if (rc) return stats->status = rc;
  c->ctl_h->nneg = c->ctl_h->nnonfinite = c->ctl_h->nwasted = 0;
  c->ctl_h->icordry = 0;
  c->ctl_h->counter = 0;
  if ((rc = write_ctl(c))) return stats->status = rc;

  // time levels by buffer swap: after it the *1 buffers hold the entry values
  // (UHDY1E=UHDYE, VHDX1E=VHDXE, H1P=HP, calpuv2c.f90:256-264) and the
  // others are rewritten for every water cell before they are read
  std::swap(c->X.uhdye, c->X.uhdy1e);
  std::swap(c->X.vhdxe, c->X.vhdx1e);
  std::swap(c->X.hp, c->X.h1p);
  xm::launch_begin(c->L(), c->S, c->X, s);
  if (prm->isdry > 0) xm::launch_obc_reset(l, c->B, c->X);
  CK(cudaGetLastError());
  int ncordry = 0, status = EFDC_XM_OK;
  for (;;) {  // 1000 CONTINUE
    xm::launch_assemble(l, c->S, c->X, s, c->ctl, c->part);
    xm::launch_obc(l, c->S, c->X, c->B, s, c->ctl, c->obc_serial);
    xm::launch_scale(l, c->S, c->X, c->Y, c->ctl, mixed ? 1 : 0, c->may_asym ? 1 : 0);
    CK(cudaGetLastError());
    int iters = 0, st = 0, outer = 0;
    double rsq = 0;
    rc = mixed ? solve_mixed(c, c->X.p, prm->rsqm, prm->iterm, &iters, &rsq, &st, &outer,
                             prm->mixed_rsq_factor)
               : solve_fp64(c, c->X.p, prm->rsqm, prm->iterm, &iters, &rsq, &st);
    if (rc) return stats->status = rc;
    if (c->ctl_h->asym & 2) {
      set_error("the scaled operator is unsymmetric although the model has no radiation "
                "boundary (check SUBO/SVBO next to the open-boundary cells)");
      return stats->status = EFDC_XM_UNSUPPORTED;
    }
    stats->iters_last = iters;
    stats->iters_total += iters;
    stats->solves += 1;
    stats->rsq_last = rsq;
    stats->outer_refinements += outer;
    stats->ccmnm_last = std::min(c->ctl_h->ccmnm_int, c->ctl_h->ccmnm_bc);
    if (st != EFDC_XM_OK) {
      status = st;
      set_error("CONGRAD: %s after %d iterations (RSQ=%g, RSQM=%g)",
                st == EFDC_XM_CG_MAXITER ? "maximum iterations exceeded" : "non-finite residual",
                iters, rsq, prm->rsqm);
      break;
    }
    xm::launch_backsub(l, c->S, c->X, s);
    xm::launch_obc_hp(l, c->S, c->X, c->B, s);
    if (prm->isdry > 0 && prm->isdry < 98) {
      xm::launch_wd_legacy(l, c->S, c->X, s, c->ctl, 1);
    } else if (prm->isdry == 99) {
      xm::launch_wd99(l, c->S, c->X, s, c->ctl);
    } else if (prm->isdry > 0) {
      xm::launch_wd_legacy(l, c->S, c->X, s, c->ctl, 0);
    }
    CK(cudaGetLastError());
    if (prm->isdry > 0 && prm->isdry != 98) {
      if ((rc = read_ctl(c))) return stats->status = rc;
      if (c->ctl_h->icordry) {
        c->ctl_h->icordry = 0;
        if ((rc = write_ctl(c))) return stats->status = rc;
        ++ncordry;
        if (ncordry < max_sweeps) continue;
        status = EFDC_XM_WETDRY_MAXSWEEP;
        set_error("wet/dry: NCORDRY reached %d", max_sweeps);
        break;
      }
    }
    break;
  }
  if (status == EFDC_XM_OK) {
    xm::launch_final(l, c->S, c->X, s, c->ctl);
    CK(cudaGetLastError());
  }
  if ((rc = read_ctl(c))) return stats->status = rc;
  stats->n_negdep = c->ctl_h->nneg;
  stats->n_wasted = c->ctl_h->nwasted;
  if (status == EFDC_XM_OK && c->ctl_h->nnonfinite > 0) {
    status = EFDC_XM_NONFINITE;
    set_error("non-finite P in %d cells", c->ctl_h->nnonfinite);
  }
  if (status == EFDC_XM_OK && c->ctl_h->nneg > 0) status = EFDC_XM_NEG_DEPTH;
  stats->status = status;
  return status;
}

int32_t efdc_xm_step(efdc_xm_ctx *c, const efdc_xm_params *prm, efdc_xm_fields *f,
                     efdc_xm_stats *stats) {
  efdc_xm_stats dummy;
  if (!stats) stats = &dummy;
  std::memset(stats, 0, sizeof(*stats));
  if (!c || !prm || !f || !f->p || !f->hp || !f->hu || !f->hv || !f->uhdye || !f->vhdxe ||
      !f->sub || !f->svb) {
    set_error("efdc_xm_step: NULL argument (P, HP, HU, HV, UHDYE, VHDXE, SUB, SVB are required)");
    return stats->status = EFDC_XM_BAD_ARGUMENT;
  }
  if (prm->isdry > 0 && (!f->sbx || !f->sby || !f->lmaskdry || !f->iscdry)) {
    set_error("efdc_xm_step: ISDRY>0 needs SBX, SBY, LMASKDRY and ISCDRY");
    return stats->status = EFDC_XM_BAD_ARGUMENT;
  }
  int rc = efdc_xm_upload(c, f);
  if (rc) return stats->status = rc;
  const int st = efdc_xm_step_device(c, prm, stats);
  if (st == EFDC_XM_CUDA_ERROR || st == EFDC_XM_BAD_ARGUMENT) return st;
  rc = efdc_xm_download(c, f);
  if (rc) return stats->status = rc;
  if (f->lwet || f->ldry) {
    if (prm->isdry == 0) {
      stats->lawet = c->la - 1;
      stats->ladry = 0;
    } else {
      int nw = 0, nd = 0;
      for (int L = 2; L <= c->la; ++L) {
        if (f->lmaskdry[L - 1]) ++nw;
        else if ((!c->oldmask_h.empty() && c->oldmask_h[L - 1]) || prm->n < prm->ntstbc + 1) ++nd;
      }
      stats->lawet = nw;
      stats->ladry = nd;
    }
  }
  return st;
}

int32_t efdc_xm_congrad(efdc_xm_ctx *c, const double *ccc, const double *ccs, const double *ccn,
                        const double *ccw, const double *cce, const double *ccci,
                        const double *fptmp, double *p, double rsqm, int32_t iterm,
                        int32_t precision, int32_t *iters, double *rsq) {
  if (!c || !ccc || !ccs || !ccn || !ccw || !cce || !fptmp || !p || iterm < 1) {
    set_error("efdc_xm_congrad: NULL argument or ITERM < 1");
    return EFDC_XM_BAD_ARGUMENT;
  }
  (void)ccci;  // CCCI = 1./CCC is recomputed on the device (same rounding)
  CK(cudaSetDevice(c->device));
  // the scaled system; land slots are reset to the inert CCC=1, C*=0, b=0
  std::vector<Xfer> xs = {{ccc, c->Y.ccc, 3}, {ccs, c->Y.ccs, 3}, {ccn, c->Y.ccn, 3},
                          {ccw, c->Y.ccw, 3}, {cce, c->Y.cce, 3}, {fptmp, c->Y.fptmp, 3},
                          {p, c->X.p, 0}};
  int rc = upload_arrays(c, xs);
  if (rc) return rc;
  CK(cudaMemsetAsync(&c->ctl->asym, 0, sizeof(int), c->stream));
  xm::launch_sys_prepare(c->L(), c->S, c->Y, c->ctl, precision == EFDC_XM_PREC_MIXED ? 1 : 0);
  CK(cudaGetLastError());
  int it = 0, st = 0, outer = 0;
  double r = 0;
  rc = (precision == EFDC_XM_PREC_MIXED)
           ? solve_mixed(c, c->X.p, rsqm, iterm, &it, &r, &st, &outer, 0.0)
           : solve_fp64(c, c->X.p, rsqm, iterm, &it, &r, &st);
  if (rc) return rc;
  std::vector<Xfer> out = {{p, c->X.p, 0}};
  rc = download_arrays(c, out);
  if (rc) return rc;
  if (iters) *iters = it;
  if (rsq) *rsq = r;
  if (st != EFDC_XM_OK)
    set_error("CONGRAD: %s after %d iterations (RSQ=%g)",
              st == EFDC_XM_CG_MAXITER ? "maximum iterations exceeded" : "non-finite residual", it, r);
  return st;
}

void *efdc_xm_stream(efdc_xm_ctx *c) { return c ? static_cast<void *>(c->stream) : nullptr; }

int64_t efdc_xm_kernel_launches(void) { return g_launches.load(); }

int32_t efdc_xm_time_kernels(efdc_xm_ctx *c, int32_t precision, int32_t reps, efdc_xm_ktime *out) {
  if (!c || !out || reps < 1 || reps > 40) {
    set_error("efdc_xm_time_kernels: need a context, an output and 1 <= reps <= 40");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  const xm::Launch l = c->L();
  cudaEvent_t ev[3];
  for (auto &e : ev) CK(cudaEventCreate(&e));
  double tm = 0, tu = 0;
  // the iterations run on a scratch copy of P with the stop test disabled
  CK(cudaMemcpyAsync(c->ptmp, c->X.p, size_t(c->nslot) * sizeof(double), cudaMemcpyDeviceToDevice,
                     c->stream));
  if (precision == EFDC_XM_PREC_MIXED) {
    xm::launch_mx_resid(l, c->S, c->Y, c->ptmp, c->ctl, c->part, 0.0, 0.0);
  } else {
    xm::launch_cg_init(l, c->S, c->Y, c->ptmp, c->ctl, c->part);
  }
  CK(cudaGetLastError());
  int rc = read_ctl(c);
  if (rc) return rc;
  c->ctl_h->done = 0;
  c->ctl_h->idone = 0;
  c->ctl_h->status = 0;
  if ((rc = write_ctl(c))) return rc;
  for (int k = 0; k < reps; ++k) {
    CK(cudaEventRecord(ev[0], c->stream));
    if (precision == EFDC_XM_PREC_MIXED) {
      xm::launch_mx_matvec(l, c->S, c->Y, c->ctl, c->part);
      CK(cudaEventRecord(ev[1], c->stream));
      xm::launch_mx_update(l, c->S, c->Y, c->ctl, c->part, INT_MAX, INT_MAX);
    } else {
      xm::launch_cg_matvec(l, c->S, c->Y, c->ctl, c->part);
      CK(cudaEventRecord(ev[1], c->stream));
      xm::launch_cg_update(l, c->S, c->Y, c->ptmp, c->ctl, c->part, -1.0, INT_MAX);
    }
    CK(cudaEventRecord(ev[2], c->stream));
    CK(cudaEventSynchronize(ev[2]));
    float a = 0, b = 0;
    CK(cudaEventElapsedTime(&a, ev[0], ev[1]));
    CK(cudaEventElapsedTime(&b, ev[1], ev[2]));
    tm += a;
    tu += b;
  }
  if ((rc = read_ctl(c))) return rc;
  for (auto &e : ev) cudaEventDestroy(e);
  out->ms_matvec = tm / reps;
  out->ms_update = tu / reps;
  out->reps = reps;
  out->ncells = c->la - 1;
  out->nslots = (c->ntile - 1) * TILE;
  if (c->ctl_h->done) {
    set_error("efdc_xm_time_kernels: the iteration stopped early (status %d)", c->ctl_h->status);
    return EFDC_XM_NONFINITE;
  }
  return EFDC_XM_OK;
}

}  // extern "C"
