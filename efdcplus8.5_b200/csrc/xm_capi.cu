// xm_capi.cu -- the C-ABI of libefdc_xm (include/efdc_xm.h): context set-up
// (tile layout of M >= 1 basins, device arrays), host<->device transfers, and
// the host-side orchestration of one CALPUV2C step (calpuv2c.f90:128-1187) of
// every member and of CONGRAD.

#include <algorithm>
#include <array>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_set>
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
std::atomic<long long> g_h2d{0}, g_d2h{0};  // bytes of the callers' arrays copied
std::atomic<long long> g_waits{0};  // host waits for the device inside step and solve calls

using xm::CopyJob;
using xm::Ctl;
using xm::Glob;
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

constexpr int NSTAGE = 8;     // staging buffers (each holds one array of every member)
constexpr int NCHUNK = 32;    // most member chunks of a pipelined efdc_xm_step_batch
constexpr int NCOPY = 4;      // streams for host<->device copies
// Contexts of at most this many members fold the member reductions into the
// CG kernels by default.  In a larger batch the CTA that stores last often
// completes many members at once and sums them one after another at the end
// of the kernel (measured on 256 members: the inner iteration's kernels 40-60 %
// slower), where one member-reduce kernel sums them all in parallel.
constexpr int FOLD_MEMBERS = 4;
constexpr int MAX_JOBS = 128;  // arrays moved by one upload/download call
constexpr int GRAPH_ITERS = 4;  // CG iterations per graph launch
constexpr int KERNELS_PER_ITER = 4;  // matvec, its reduce, update, its reduce

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

// One basin of the context.
// the control blocks move as 4-byte words (launch_words)
static_assert(sizeof(Ctl) % 4 == 0 && sizeof(Glob) % 4 == 0 &&
                  sizeof(xm::StepScalars) % 4 == 0,
              "control blocks must be whole 4-byte words");

struct Member {
  int la = 0, lc = 0;
  int tile0 = 0, tile1 = 0;  // its tiles [tile0, tile1); tile0 - 1 is its ghost tile
  long long off = 0;         // element offset of its arrays in the staging buffers
  int nobc = 0, b0 = 0;      // its open-boundary cells [b0, b0+nobc) of the packed list
  int side_n[4] = {0, 0, 0, 0};
  int mtide = 0;
  std::vector<double> tcp;
  bool may_asym = false;  // a radiation boundary: the operator can be unsymmetric
  int last_iters = 8, last_inner = 8;
  float jac_est = 20.f;  // Jacobi-equivalent inner iterations per outer pass (MIXED)
  int last_n = 0, last_ntstbc = 0, last_isdry = 0;
  std::vector<int32_t> oldmask_h;
  std::vector<int> slot_of;  // slot of cell L (0 for L outside 2..LA)
  // CALEXP2T's type-2 open boundaries (calexp2t.f90:605-645), W, E, S, N in
  // list order: (side, L of the modified cell, its neighbour the form reads
  // (LNC for W, LWC for E, LEC for S, LSC for N), 0)
  std::vector<int4> t2;
};

// A step captured as one graph (see step_graph): the bytes it was built from
// (flags and every device view its kernels take), and the kernels it
// launches outside its loops and per body of each loop, for the launch count.
struct StepGraph {
  std::vector<char> key;
  cudaGraphExec_t exec = nullptr;
  long long n_top = 0;
  long long n_body[xm::NLOOP] = {};
};

// One sub-grid channel of a member, as efdc_xm_set_channels received it.
struct ChanSpec {
  int type, lh, lu, lv;  // MDCHTYP, LMDCHH, LMDCHU, LMDCHV
  double len, fric;      // CHANLEN, CHANFRIC
  double gw, gl;         // guest's WCHAN and cross length (DXP/DYP of LMDCHU or LMDCHV)
};

struct efdc_xm_ctx {
  int device = 0;
  int M = 0;
  std::vector<Member> mem;
  int ntile = 0, nslot = 0, nquad = 0;
  int grid = 1, grid_cg = 1, grid_cg32 = 1, grid_up32 = 1, nsm = 0;
  long long stage_len = 0;  // elements of one staging buffer
  cudaStream_t stream = nullptr;
  // host<->device copies: many per-member copies of small arrays run
  // concurrently on NCOPY streams (each ordered after the kernels that
  // filled or before the kernels that read the staging buffers, by events)
  cudaStream_t copy_stream[NCOPY] = {};
  cudaEvent_t copy_event[NCOPY + 1] = {};
  // pipelined efdc_xm_step_batch (member chunks: the upload of one, the step
  // of another and the download of a third overlap): the download copy
  // streams, the scatter and gather streams, and events per chunk
  cudaStream_t dn_stream[NCOPY] = {};
  cudaStream_t up_x = nullptr, dn_x = nullptr;
  cudaEvent_t ev_start = nullptr, ev_up[NCHUNK] = {}, ev_step[NCHUNK] = {}, ev_g[NCHUNK] = {};
  cudaEvent_t ev_j[NCHUNK][NCOPY] = {};
  std::vector<DevBuf> bufs;
  // device views
  xm::DevStatic S{};
  xm::DevState X{};
  xm::DevSystem Y{};
  xm::DevObc B{};
  Ctl *ctl = nullptr;                // [M]
  Ctl *ctl_h = nullptr;              // [M] pinned mirror
  Glob *glob = nullptr;
  Glob *glob_h = nullptr;            // pinned
  int *act = nullptr;                // [M] member takes part in the current sweep
  int *mpoly = nullptr;              // [M] MIXED inner preconditioner of the member
  int *mpoly_h = nullptr;            // [M] pinned
  int *act_h = nullptr;              // [M] pinned
  xm::StepScalars *sc = nullptr;     // [M]
  xm::StepScalars *sc_h = nullptr;   // [M] pinned
  // device addresses of the mapped pinned mirrors (null: copied by the copy engines)
  void *ctl_hd = nullptr, *glob_hd = nullptr, *act_hd = nullptr, *mpoly_hd = nullptr,
       *sc_hd = nullptr;
  bool in_chunks = false;  // inside a chunked efdc_xm_step_batch (see to_device)
  double *part = nullptr;
  int *lidx = nullptr;
  int *tile_member = nullptr;
  long long *moff = nullptr;
  int *mlc = nullptr;
  std::vector<double *> stage;
  CopyJob *jobs_d = nullptr;
  CopyJob *jobs_h = nullptr;  // pinned
  bool obc_serial = false;
  bool any_may_asym = false;
  int nobc = 0;
  double *pser_d = nullptr;
  double *pser_h = nullptr;  // pinned
  double *ptmp = nullptr;    // scratch P for kernel timing
  double *ptune = nullptr;   // the autotuner's copy of P (allocated on first use)
  // CUDA graphs of GRAPH_ITERS consecutive CG iterations on X.p (FP64) and
  // of the FP32 inner iteration, captured on first use
  // CG iteration graphs: [may_asym | chan << 1] (FP64),
  // [kinds | may_asym << 2 | chan << 3] (MIXED)
  cudaGraphExec_t graph_cg[4] = {}, graph_mx[16] = {};
  bool graph_cg_failed[4] = {}, graph_mx_failed[16] = {};
  // device-driven steps: the whole step as one graph whose loops are
  // conditional WHILE nodes (StepGraph), cached by what the graph holds
  bool device_loops = true;     // efdc_xm_set_option(EFDC_XM_OPT_DEVICE_LOOPS)
  bool stepped = false;         // a step of every member has assembled the systems
  int graph_iters = GRAPH_ITERS;  // CG iterations per loop body
  std::vector<StepGraph> step_graphs;
  std::vector<std::vector<char>> step_graph_failed;
  cudaStream_t cap_stream[4] = {};  // capture streams of the nested loop bodies
  bool mx_jac = true, mx_poly = false;  // kinds of MIXED inner solve in use
  xm::SysView mxview{};  // the system the MIXED solve refines (the step's assembly, or CONGRAD's)
  bool last_mixed = false;  // the last step ran MIXED: the scaled FP64 system is formed on request
  bool sys_external = false;  // the system being solved is a caller's (efdc_xm_congrad)
  // calibration (efdc_xm_calib_*): adjoint state, step-start snapshots,
  // the CG solution of the last step, gauge gathers
  bool calib = false;
  xm::DevCalib A{};
  std::vector<std::array<double *, 6>> snap;  // P, HP, HU, HV, UHDYE, VHDXE
  double *psol = nullptr;
  double *bsq = nullptr;
  int *gslot = nullptr;   // [gcap] gauge slots
  double *gbuf = nullptr; // [gcap] gauge values / adjoint weights
  int gcap = 0;
  // sub-grid channels: each member's list, the slot kinds as created, and
  // the device arrays behind S.ch (rebuilt by efdc_xm_set_channels)
  std::vector<std::vector<ChanSpec>> chans;
  std::vector<uint8_t> kind_h;
  std::vector<void *> chan_bufs;
  std::vector<double> hp1_h;  // [M] HP(1) at the last upload
  std::vector<int> chan_start;  // [M+1] first channel of each member in S.ch
  std::vector<int> qstart_h;    // [M+1] first quad of each member
  double *chan_hp1 = nullptr;   // S.ch.hp1
  // baroclinic terms: layers set by efdc_xm_set_layers (S.baro), and whether
  // the current step has a member with them
  std::vector<char> has_layers;  // [M]
  bool step_baro = false;
  std::vector<double> zeros_h;   // LC zeros: B of a member without it
  // the device copies of LMASKDRY, ISCDRY, NATDRY, QDWASTE, VDWASTE (wd_stale)
  // and of SBX, SBY (sbxy_stale) are out of date: the last efdc_xm_step_batch
  // ran without wetting and drying (and without baroclinic terms) and did
  // not upload them; the host holds them
  bool wd_stale = false, sbxy_stale = false;
  // arrays (bits of enum efdc_xm_same) whose device copy is still what the
  // caller's array held at its last upload or received at its last download
  uint32_t synced = 0;
  // three time levels (CALPUV9C): their buffers are allocated by the first
  // upload that carries them (tl3_alloc); tl3_ready: the device holds a
  // consistent set of levels (uploaded, or advanced by CALPUV9C steps)
  bool tl3_alloc = false, tl3_ready = false;
  // implicit drag inputs (X.ubot ... X.fyvege): allocated by the first upload
  // that carries one; drag_in: bits of those uploaded (DRAG_*)
  bool drag_alloc = false;
  unsigned drag_in = 0;
  // bottom-stress producer (efdc_xm_set_bed, efdc_xm_bottom_stress_batch)
  xm::DevBed bed{};
  bool bed_alloc = false;
  // explicit momentum producer (efdc_xm_set_momentum): device arrays, the
  // per-member layer count and leading dimension, the serial lists
  bool mom_alloc = false;
  int mom_kc = 0;
  xm::MomDev md{};
  double *mom_hp = nullptr;
  void *mom_lists = nullptr;  // the serial lists on the device (rebuilt after a set-up call)
  char *pack_h = nullptr, *pack_d = nullptr;  // packed small transfers (page-locked, device)
  bool mom_inputs = false;    // a call has left U, V, UHDY, VHDX on the device
  std::vector<char> has_mom;
  std::vector<int> mom_ld;
  std::vector<std::vector<int4>> mom_t2, mom_bc;
  std::vector<xm::MomScalars> mom_sc_h;
  std::vector<char> has_bed;         // [M]
  std::vector<xm::DragScalars> bed_sc;  // [M] the bed's scalars (delt ... filled per call)
  xm::DragScalars *ds = nullptr;     // [M] device

  template <class T>
  T *alloc(size_t n, bool zero = true) {
    DevBuf b;
    b.bytes = std::max<size_t>(n, 1) * sizeof(T);
    if (cudaMalloc(&b.p, b.bytes) != cudaSuccess) return nullptr;
    if (zero) cudaMemset(b.p, 0, b.bytes);
    bufs.push_back(b);
    return static_cast<T *>(b.p);
  }
  // schedule of the FP32 CG kernels (efdc_xm_set_option: variant and CTA caps)
  int kvariant = 0, ctas_mv = 0, ctas_up = 0;
  int inner_margin_log10 = 0;   // MIXED inner target margin 10^-v
  int inner_tol_x10 = 60;       // MIXED inner relative tolerance 10^(-v/10) at least
  bool small_solve = true;      // FP64: members small enough solve in one CTA each
  int fold_reduce = 1;          // member reductions folded into the CG kernels:
                                // 0 never, 1 up to FOLD_MEMBERS members, 2 always
  int nchunk = 8;               // member chunks of a pipelined efdc_xm_step_batch
  int small_slots = 0;          // the largest member window (its ghost tile and tiles)
  int small_units = 0;          // the most 4-tile units of a member
  float poly_threshold = 10.f;  // MIXED: polynomial preconditioner above this Jacobi count
  xm::Launch L() const {
    xm::Launch l{grid,      grid_cg, grid_cg32, grid_up32,
                 ntile,     nsm,     stream,
                 mx_jac,  mx_poly, any_may_asym || sys_external,
                 S.ch.n > 0 && !sys_external, step_baro && !sys_external};
    l.variant = kvariant;
    l.ctas_mv = ctas_mv;
    l.ctas_up = ctas_up;
    l.inner_margin = std::pow(10.0, -double(inner_margin_log10));
    l.fold = (fold_reduce == 2 || (fold_reduce == 1 && M <= FOLD_MEMBERS)) && !l.chan;
    return l;
  }
};

namespace {

// Transfer plan entry: one array of every member (host pointers, element L
// at [L-1], LC elements) and the tile-order device array.
struct Xfer {
  std::vector<const void *> host;  // [M]
  void *dev;
  int kind;  // 0 double, 1 LOGICAL (normalised to 0/1), 2 raw int, 3 double water-only
};

size_t esize(int kind) { return (kind == 1 || kind == 2) ? sizeof(int32_t) : sizeof(double); }

// A field moves when every member gives it; given for some members only, it is an error.
int collect(efdc_xm_ctx *c, std::vector<Xfer> &out, const std::vector<const void *> &ptrs,
            const void *dev, int kind, const char *name) {
  int n = 0;
  for (const void *p : ptrs) n += p ? 1 : 0;
  if (n == 0 || !dev) return EFDC_XM_OK;
  if (n != c->M) {
    set_error("field %s is given for %d of %d members (all or none)", name, n, c->M);
    return EFDC_XM_BAD_ARGUMENT;
  }
  out.push_back(Xfer{ptrs, const_cast<void *>(dev), kind});
  return EFDC_XM_OK;
}

// The copy streams wait for the compute stream's work so far, and the compute
// stream then waits for the copies issued on them.
int copies_after_compute(efdc_xm_ctx *c) {
  CK(cudaEventRecord(c->copy_event[NCOPY], c->stream));
  for (cudaStream_t s : c->copy_stream) CK(cudaStreamWaitEvent(s, c->copy_event[NCOPY], 0));
  return EFDC_XM_OK;
}
int compute_after_copies(efdc_xm_ctx *c) {
  for (int k = 0; k < NCOPY; ++k) {
    CK(cudaEventRecord(c->copy_event[k], c->copy_stream[k]));
    CK(cudaStreamWaitEvent(c->stream, c->copy_event[k], 0));
  }
  return EFDC_XM_OK;
}

// Host -> staging copies of the members [m0, m1) of one array (members whose
// host arrays lie back to back at the staging stride, LC+1 elements -- an
// ensemble held as one (LCM, members) array per field -- go in one copy),
// spread over the streams st[k++ % NCOPY].
int h2d_range(efdc_xm_ctx *c, const Xfer &x, char *stage, int m0, int m1, cudaStream_t *st,
              int &k, int ns = NCOPY) {
  const size_t es = esize(x.kind);
  for (int m = m0; m < m1;) {
    const char *h0 = static_cast<const char *>(x.host[m]);
    int e = m + 1;
    while (e < m1 && static_cast<const char *>(x.host[e]) ==
                         static_cast<const char *>(x.host[e - 1]) +
                             size_t(c->mem[e - 1].lc + 1) * es)
      ++e;
    const size_t n = size_t(c->mem[e - 1].off - c->mem[m].off + c->mem[e - 1].lc);
    CK(cudaMemcpyAsync(stage + c->mem[m].off * es, h0, n * es, cudaMemcpyHostToDevice,
                       st[k++ % ns]));
    g_h2d.fetch_add(static_cast<long long>(n * es), std::memory_order_relaxed);
    m = e;
  }
  return EFDC_XM_OK;
}

// A caller's host element that a staging -> host copy overwrites and that is
// put back once the copy is done.
struct Keep {
  char *at;
  char val[8];
  size_t n;
};

// Staging -> host copies of the members [m0, m1) of one array.  A member
// alone sends its water elements L = 2..LA; members back to back at the
// staging stride go in one copy of the whole run, which also covers each
// member's ghost elements (L = 1 and LC) and the element between two members:
// those must stay as the caller has them, so their values go to `keep`.
int d2h_range(efdc_xm_ctx *c, const Xfer &x, const char *stage, int m0, int m1, cudaStream_t *st,
              int &k, std::vector<Keep> &keep, int ns = NCOPY) {
  const size_t es = esize(x.kind);
  auto save = [&](char *at) {
    Keep kp{at, {}, es};
    std::memcpy(kp.val, at, es);
    keep.push_back(kp);
  };
  for (int m = m0; m < m1;) {
    char *h0 = static_cast<char *>(const_cast<void *>(x.host[m]));
    int e = m + 1;
    while (e < m1 && static_cast<const char *>(x.host[e]) ==
                         static_cast<const char *>(x.host[e - 1]) +
                             size_t(c->mem[e - 1].lc + 1) * es)
      ++e;
    if (e == m + 1) {
      const size_t n = es * size_t(c->mem[m].la - 1);
      CK(cudaMemcpyAsync(h0 + es, stage + (c->mem[m].off + 1) * es, n, cudaMemcpyDeviceToHost,
                         st[k++ % ns]));
      g_d2h.fetch_add(static_cast<long long>(n), std::memory_order_relaxed);
    } else {
      for (int q = m; q < e; ++q) {
        char *hq = static_cast<char *>(const_cast<void *>(x.host[q]));
        save(hq);                                              // L = 1
        save(hq + size_t(c->mem[q].lc - 1) * es);              // L = LC
        if (q + 1 < e) save(hq + size_t(c->mem[q].lc) * es);   // between members
      }
      const size_t n = es * size_t(c->mem[e - 1].off - c->mem[m].off + c->mem[e - 1].lc);
      CK(cudaMemcpyAsync(h0, stage + c->mem[m].off * es, n, cudaMemcpyDeviceToHost,
                         st[k++ % ns]));
      g_d2h.fetch_add(static_cast<long long>(n), std::memory_order_relaxed);
    }
    m = e;
  }
  return EFDC_XM_OK;
}

// Small transfers (the fields of small basins): the call's arrays go through
// one page-locked host buffer and one device buffer, a host copy per array and
// member, one copy over the link and one scatter (or one gather, one copy back
// and host copies out).  A few link operations per call instead of one per
// array: those, not bytes, bound a small basin's step on host arrays.
constexpr size_t PACK_MAX = size_t(4) << 20;  // bytes of one packed transfer

bool packed(efdc_xm_ctx *c, size_t njobs) {
  const size_t bytes = njobs * size_t(c->stage_len) * sizeof(double);
  if (bytes > PACK_MAX) return false;
  if (!c->pack_h) {
    if (cudaHostAlloc(&c->pack_h, PACK_MAX, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      c->pack_h = nullptr;
      return false;
    }
    if (!(c->pack_d = c->alloc<char>(PACK_MAX, false))) {
      cudaFreeHost(c->pack_h);
      c->pack_h = nullptr;
      return false;
    }
  }
  return true;
}

int upload_packed(efdc_xm_ctx *c, const std::vector<Xfer> &xs) {
  const size_t L = size_t(c->stage_len), n = xs.size();
  for (size_t j = 0; j < n; ++j) {
    const size_t es = esize(xs[j].kind);
    char *dst = c->pack_h + j * L * sizeof(double);
    for (int m = 0; m < c->M; ++m)
      if (xs[j].host[m])
        std::memcpy(dst + size_t(c->mem[m].off) * es, xs[j].host[m], size_t(c->mem[m].lc) * es);
    c->jobs_h[j] = CopyJob{reinterpret_cast<double *>(c->pack_d + j * L * sizeof(double)),
                           xs[j].dev, xs[j].kind};
  }
  const size_t bytes = n * L * sizeof(double);
  CK(cudaMemcpyAsync(c->jobs_d, c->jobs_h, n * sizeof(CopyJob), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaMemcpyAsync(c->pack_d, c->pack_h, bytes, cudaMemcpyHostToDevice, c->stream));
  g_h2d.fetch_add(static_cast<long long>(bytes), std::memory_order_relaxed);
  xm::launch_scatter(c->stream, c->jobs_d, int(n), c->lidx, c->tile_member, c->moff, c->mlc, 0,
                     c->nslot);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));  // the host buffer is reused by the next call
  return EFDC_XM_OK;
}

int download_packed(efdc_xm_ctx *c, const std::vector<Xfer> &xs) {
  const size_t L = size_t(c->stage_len), n = xs.size();
  for (size_t j = 0; j < n; ++j)
    c->jobs_h[j] = CopyJob{reinterpret_cast<double *>(c->pack_d + j * L * sizeof(double)),
                           xs[j].dev, xs[j].kind};
  const size_t bytes = n * L * sizeof(double);
  CK(cudaMemcpyAsync(c->jobs_d, c->jobs_h, n * sizeof(CopyJob), cudaMemcpyHostToDevice,
                     c->stream));
  xm::launch_gather(c->stream, c->jobs_d, int(n), c->lidx, c->tile_member, c->moff, 0, c->nslot);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->pack_h, c->pack_d, bytes, cudaMemcpyDeviceToHost, c->stream));
  g_d2h.fetch_add(static_cast<long long>(bytes), std::memory_order_relaxed);
  CK(cudaStreamSynchronize(c->stream));
  for (size_t j = 0; j < n; ++j) {  // the water elements L = 2..LA of each member
    const size_t es = esize(xs[j].kind);
    const char *src = c->pack_h + j * L * sizeof(double);
    for (int m = 0; m < c->M; ++m)
      if (xs[j].host[m])
        std::memcpy(static_cast<char *>(const_cast<void *>(xs[j].host[m])) + es,
                    src + size_t(c->mem[m].off + 1) * es, size_t(c->mem[m].la - 1) * es);
  }
  return EFDC_XM_OK;
}

int upload_arrays(efdc_xm_ctx *c, const std::vector<Xfer> &xs) {
  if (xs.empty()) return EFDC_XM_OK;
  if (xs.size() > size_t(MAX_JOBS)) {
    set_error("internal: too many arrays in one transfer");
    return EFDC_XM_CUDA_ERROR;
  }
  if (packed(c, xs.size())) return upload_packed(c, xs);
  for (size_t j = 0; j < xs.size(); ++j)
    c->jobs_h[j] = CopyJob{c->stage[j % NSTAGE], xs[j].dev, xs[j].kind};
  CK(cudaMemcpyAsync(c->jobs_d, c->jobs_h, xs.size() * sizeof(CopyJob), cudaMemcpyHostToDevice,
                     c->stream));
  int rc = 0, k = 0;
  for (size_t g0 = 0; g0 < xs.size(); g0 += NSTAGE) {
    const size_t g1 = std::min(xs.size(), g0 + NSTAGE);
    // the previous group's scatter has read the staging buffers
    if ((rc = copies_after_compute(c))) return rc;
    for (size_t j = g0; j < g1; ++j)
      if ((rc = h2d_range(c, xs[j], reinterpret_cast<char *>(c->stage[j % NSTAGE]), 0, c->M,
                          c->copy_stream, k)))
        return rc;
    if ((rc = compute_after_copies(c))) return rc;
    xm::launch_scatter(c->stream, c->jobs_d + g0, int(g1 - g0), c->lidx, c->tile_member, c->moff,
                       c->mlc, 0, c->nslot);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(c->stream));
  return EFDC_XM_OK;
}

int download_arrays(efdc_xm_ctx *c, const std::vector<Xfer> &xs) {
  if (xs.empty()) return EFDC_XM_OK;
  if (xs.size() > size_t(MAX_JOBS)) {
    set_error("internal: too many arrays in one transfer");
    return EFDC_XM_CUDA_ERROR;
  }
  if (packed(c, xs.size())) return download_packed(c, xs);
  for (size_t j = 0; j < xs.size(); ++j)
    c->jobs_h[j] = CopyJob{c->stage[j % NSTAGE], xs[j].dev, xs[j].kind};
  CK(cudaMemcpyAsync(c->jobs_d, c->jobs_h, xs.size() * sizeof(CopyJob), cudaMemcpyHostToDevice,
                     c->stream));
  std::vector<Keep> keep;  // put back once the copies are done (the caller waits here)
  int rc = 0, k = 0;
  for (size_t g0 = 0; g0 < xs.size(); g0 += NSTAGE) {
    const size_t g1 = std::min(xs.size(), g0 + NSTAGE);
    if (g0 > 0 && (rc = compute_after_copies(c))) return rc;  // the buffers were copied out
    xm::launch_gather(c->stream, c->jobs_d + g0, int(g1 - g0), c->lidx, c->tile_member, c->moff,
                      0, c->nslot);
    CK(cudaGetLastError());
    if ((rc = copies_after_compute(c))) return rc;
    for (size_t j = g0; j < g1; ++j)
      if ((rc = d2h_range(c, xs[j], reinterpret_cast<const char *>(c->stage[j % NSTAGE]), 0,
                          c->M, c->copy_stream, k, keep)))
        return rc;
  }
  for (cudaStream_t s : c->copy_stream) CK(cudaStreamSynchronize(s));
  CK(cudaStreamSynchronize(c->stream));
  for (const Keep &kp : keep) std::memcpy(kp.at, kp.val, kp.n);
  return EFDC_XM_OK;
}

// Control blocks between the device and their pinned host mirrors, on the
// solver stream.  During a chunked efdc_xm_step_batch (c->in_chunks), where
// the mirror is mapped (dev_h: its device address), a kernel moves them, so
// that a step's polls do not queue behind the bulk copies in flight on the
// copy engines; otherwise the copy engines do.
int to_device(efdc_xm_ctx *c, void *dev, const void *host, const void *dev_h, size_t bytes) {
  if (dev_h && c->in_chunks) {
    xm::launch_words(c->stream, dev, dev_h, bytes);
    CK(cudaGetLastError());
  } else {
    CK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, c->stream));
  }
  return EFDC_XM_OK;
}
int to_host(efdc_xm_ctx *c, void *host, void *dev_h, const void *dev, size_t bytes) {
  if (dev_h && c->in_chunks) {
    xm::launch_words(c->stream, dev_h, dev, bytes);
    CK(cudaGetLastError());
  } else {
    CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  g_waits.fetch_add(1, std::memory_order_relaxed);
  return EFDC_XM_OK;
}

int read_ctl(efdc_xm_ctx *c) {
  return to_host(c, c->ctl_h, c->ctl_hd, c->ctl, sizeof(Ctl) * c->M);
}

int read_glob(efdc_xm_ctx *c) {
  return to_host(c, c->glob_h, c->glob_hd, c->glob, sizeof(Glob));
}

int write_act(efdc_xm_ctx *c) {
  return to_device(c, c->act, c->act_h, c->act_hd, sizeof(int) * c->M);
}

// Captures `body` (GRAPH_ITERS iterations launched on c->stream) into a
// graph.  A failed capture leaves plain launches in use (same kernels).
template <class Body>
cudaGraphExec_t capture_graph(efdc_xm_ctx *c, Body body) {
  const long long before = g_launches.load();
  cudaGraph_t g = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  for (int k = 0; k < GRAPH_ITERS; ++k) body();
  const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  g_launches.fetch_sub(g_launches.load() - before);  // captured, not launched
  if (e != cudaSuccess || !g) {
    cudaGetLastError();
    return nullptr;
  }
  if (cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
    cudaGetLastError();
    exec = nullptr;
  }
  cudaGraphDestroy(g);
  return exec;
}

// `n` CG iterations: whole graphs where they fit, single launches for the rest.
int run_iters(efdc_xm_ctx *c, bool mixed, double *P, int n) {
  const xm::Launch l = c->L();
  // the kernels the graph holds
  const int ma = l.may_asym ? 1 : 0, ch = l.chan ? 1 : 0;
  const int kind = (c->mx_jac ? 1 : 0) | (c->mx_poly ? 2 : 0) | (ma << 2) | (ch << 3);
  cudaGraphExec_t &gr = mixed ? c->graph_mx[kind] : c->graph_cg[ma | (ch << 1)];
  bool &failed = mixed ? c->graph_mx_failed[kind] : c->graph_cg_failed[ma | (ch << 1)];
  auto one = [&]() {
    if (mixed)
      xm::launch_mx_iter(l, c->S, c->Y, c->ctl, c->glob, c->part);
    else
      xm::launch_cg_iter(l, c->S, c->Y, P, c->ctl, c->glob, c->part);
  };
  if (!gr && !failed && n >= GRAPH_ITERS && P == c->X.p) {
    gr = capture_graph(c, one);
    failed = (gr == nullptr);
  }
  int k = 0;
  if (gr && P == c->X.p) {
    for (; k + GRAPH_ITERS <= n; k += GRAPH_ITERS) {
      CK(cudaGraphLaunch(gr, c->stream));
      xm::count_launches(GRAPH_ITERS * KERNELS_PER_ITER);
    }
  }
  for (; k < n; ++k) one();
  CK(cudaGetLastError());
  return EFDC_XM_OK;
}

// The scaled FP64 system of the last step (calpuv2c.f90:371-399), which a
// MIXED step does not form itself; for downloads and FP64 kernel timing.
int scaled_system(efdc_xm_ctx *c) {
  for (int m = 0; m < c->M; ++m) c->act_h[m] = 1;
  int rc = write_act(c);
  if (rc) return rc;
  xm::launch_scale(c->L(), c->S, c->X, c->Y, c->ctl, c->act, 0, 1);
  CK(cudaGetLastError());
  c->last_mixed = false;
  return EFDC_XM_OK;
}

// FP64 CONGRAD of every active member on the scaled system in c->Y.  The
// members iterate in lockstep launches; a member that has stopped is skipped
// by the kernels.  On return c->ctl_h holds each member's outcome.
// FP64 solves in one CTA per member (k_cg_small): every member's window fits
// in a CTA's shared memory and no member has sub-grid channels (their terms
// are separate kernels of the multi-kernel CG).
bool small_solve(const efdc_xm_ctx *c) {
  return c->small_solve && c->small_slots > 0 && xm::cg_small_fits(c->small_slots) &&
         c->S.ch.n == 0;
}

int solve_fp64(efdc_xm_ctx *c, double *P) {
  const xm::Launch l = c->L();
  xm::launch_solve_reset(l, c->ctl, c->glob, c->act, c->M);
  if (small_solve(c)) {  // the whole CG of each member in one CTA (k_cg_small)
    xm::launch_cg_small(l, c->S, c->Y, P, c->ctl, c->glob, c->part, c->small_slots,
                        c->small_units, c->M);
    CK(cudaGetLastError());
    int rc = read_ctl(c);
    if (rc) return rc;
    for (int m = 0; m < c->M; ++m) {
      if (!c->act_h[m]) continue;
      Ctl &k = c->ctl_h[m];
      if (!k.done && k.status == 0) k.status = EFDC_XM_CG_MAXITER;
      if (k.iter > 0) c->mem[m].last_iters = k.iter;
    }
    return EFDC_XM_OK;
  }
  xm::launch_cg_init(l, c->S, c->Y, P, c->ctl, c->glob, c->part);
  CK(cudaGetLastError());
  int chunk = 1, cap = 1;
  for (int m = 0; m < c->M; ++m)
    if (c->act_h[m]) {
      chunk = std::max(chunk, c->mem[m].last_iters);
      cap = std::max(cap, c->sc_h[m].iterm);
    }
  chunk = std::min(chunk, cap);
  int launched = 0;
  for (;;) {
    const int n = std::min(chunk, cap - launched);
    int rc = run_iters(c, false, P, n);
    if (rc) return rc;
    launched += n;
    rc = read_glob(c);
    if (rc) return rc;
    if (c->glob_h->ndone >= c->M || launched >= cap) break;
    chunk = 4;
  }
  xm::launch_cg_finish(l, c->S, c->Y, P, c->ctl);  // the last iteration's P += alpha*p
  CK(cudaGetLastError());
  int rc = read_ctl(c);
  if (rc) return rc;
  for (int m = 0; m < c->M; ++m) {
    if (!c->act_h[m]) continue;
    Ctl &k = c->ctl_h[m];
    if (!k.done && k.status == 0) k.status = EFDC_XM_CG_MAXITER;
    if (k.iter > 0) c->mem[m].last_iters = k.iter;
  }
  return EFDC_XM_OK;
}

constexpr int MAX_OUTER = 30;        // MIXED refinement passes per solve
// inner: |r| down by at least 10^(-inner_tol_x10/10) (default 1e-6; FP32 reaches ~1e-7)
double inner_rel_tol(const efdc_xm_ctx *c) { return std::pow(10.0, -0.1 * c->inner_tol_x10); }

// MIXED: each member's inner preconditioner for the next solve, and the kinds
// of inner solve the launches need; uploads the choice.  The Neumann
// polynomial halves the iterations at ~1.3x the cost of one; members whose
// Jacobi solve takes few iterations keep Jacobi.  A member whose operator
// turns out unsymmetric (its flag is set on the device) runs Jacobi whatever
// the choice, so the Jacobi kernels are launched too wherever that can
// happen: a radiation boundary, or a caller's standalone system.
int choose_inner(efdc_xm_ctx *c) {
  const xm::Launch l = c->L();
  c->mx_jac = c->mx_poly = false;
  for (int m = 0; m < c->M; ++m) {
    // a member with sub-grid channels keeps Jacobi (the couplings enter A*p only)
    c->mpoly_h[m] =
        (c->mem[m].jac_est > c->poly_threshold && !(l.chan && !c->chans[m].empty())) ? 1 : 0;
    if (!c->act_h[m]) continue;
    if (!c->mpoly_h[m]) {
      c->mx_jac = true;
    } else {
      c->mx_poly = true;
      if (c->mem[m].may_asym || c->sys_external) c->mx_jac = true;
    }
  }
  return to_device(c, c->mpoly, c->mpoly_h, c->mpoly_hd, sizeof(int) * c->M);
}

// MIXED: FP64 refinement around the FP32 inner PCG, all active members in
// lockstep outer passes.
int solve_mixed(efdc_xm_ctx *c, double *P, double factor) {
  const double fac = factor > 0 ? factor : 0.1;  // stop at fac*RSQM in FP64
  xm::launch_solve_reset(c->L(), c->ctl, c->glob, c->act, c->M);
  if (int rc0 = choose_inner(c)) return rc0;
  const xm::Launch lk = c->L();  // with the kinds in use
  xm::launch_chan_p0(lk, c->S, c->mxview, P, c->act);
  int rc = 0;
  for (int o = 0; o < MAX_OUTER; ++o) {
    xm::launch_outer_reset(lk, c->glob);
    xm::launch_mx_resid(lk, c->S, c->mxview, c->Y, P, c->ctl, c->glob, c->part, fac,
                        inner_rel_tol(c), 0);
    CK(cudaGetLastError());
    if ((rc = read_glob(c))) return rc;
    if (c->glob_h->ndone >= c->M) break;
    int chunk = 1;
    for (int m = 0; m < c->M; ++m)
      if (c->act_h[m]) chunk = std::max(chunk, c->mem[m].last_inner);
    for (int guard = 0;; ++guard) {
      if ((rc = run_iters(c, true, P, chunk))) return rc;
      if ((rc = read_glob(c))) return rc;
      if (c->glob_h->nidone + c->glob_h->ndone >= c->M) break;
      chunk = 4;
      if (guard > 100000) {  // the inner stop test caps iterations; this is a backstop
        set_error("internal: inner solve did not finish");
        return EFDC_XM_CUDA_ERROR;
      }
    }
    xm::launch_mx_apply(lk, c->S, c->mxview, c->Y, P, c->ctl);
    CK(cudaGetLastError());
    if ((rc = read_ctl(c))) return rc;
    for (int m = 0; m < c->M; ++m)
      if (c->act_h[m] && c->ctl_h[m].inner_iter > 0) {
        c->mem[m].last_inner = c->ctl_h[m].inner_iter;
        if (o == 0) {  // the first pass carries the solve
          const bool poly = c->mpoly_h[m] && !(c->ctl_h[m].asym & 1);
          c->mem[m].jac_est = float(c->ctl_h[m].inner_iter) * (poly ? 1.9f : 1.0f);
        }
      }
  }
  if ((rc = read_ctl(c))) return rc;
  for (int m = 0; m < c->M; ++m) {
    if (!c->act_h[m]) continue;
    Ctl &k = c->ctl_h[m];
    if (!k.done && k.status == 0) k.status = EFDC_XM_CG_MAXITER;
  }
  return EFDC_XM_OK;
}

xm::StepScalars make_scalars(const Member &mb, const efdc_xm_params *p) {
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
  s.max_sweeps = p->max_sweeps > 0 ? p->max_sweeps : 500;
  s.rlamn = p->qcherr;  // calpuv2c.f90:353 (RLAMN = QCHERR)
  s.baro = p->bsc > 1.E-6 ? 1 : 0;  // calpuv2c.f90:161, 192
  s.gp = p->gp;
  s.chan_consistent = p->chan_consistent != 0 ? 1 : 0;
  s.istl = p->tl3_istl;
  s.nctbc = p->nctbc;
  s.rold = p->rold;
  s.rnew = p->rnew;
  s.isitb = p->isitb;
  s.isveg = p->isveg;
  s.ritb = p->ritb;
  // setopenbc.f90:24-29 on the host, libm as the reference
  for (int m = 0; m < mb.mtide && m < xm::MT_MAX; ++m) {
    double TM = std::fmod(p->tn, mb.tcp[m]);
    TM = p->pi2 * TM / mb.tcp[m];
    s.cosv[m] = std::cos(TM);
    s.sinv[m] = std::sin(TM);
  }
  return s;
}

// Tile layout of one member on the host.
struct MemberLayout {
  std::vector<std::pair<uint64_t, int>> tiles;  // (Morton key, ty*ntx+tx), Morton order
  std::vector<int> tile_of;                     // local tile number (1-based) of (tx,ty), 0 none
  int ntx = 0, nty = 0, imin = 0, jmin = 0;
};

// Checks one member's grid (a structured grid with the reference's
// neighbour maps) and lays out its tiles.  Returns false with the error set.
bool member_layout(const efdc_xm_grid *g, int mi, MemberLayout &ml) {
  const int la = g->la, lc = g->lc;
  if (la < 2 || lc != la + 1) {
    set_error("efdc_xm_create: member %d: need LA >= 2 and LC == LA+1 (got LA=%d LC=%d)", mi, la,
              lc);
    return false;
  }
  if (!g->il || !g->jl || !g->lnc || !g->lsc || !g->lec || !g->lwc) {
    set_error("efdc_xm_create: member %d: IL, JL and the four neighbour maps are required", mi);
    return false;
  }
  const double *req[] = {g->dxyp, g->dxyip, g->dxiu, g->dyiu, g->dxiv, g->dyiv, g->dxyu, g->dxyv,
                         g->hruo, g->hrvo, g->subo, g->svbo, g->sbxo, g->sbyo, g->belv};
  for (const double *r : req)
    if (!r) {
      set_error("efdc_xm_create: member %d: a metric array is NULL", mi);
      return false;
    }
  if (g->mtide < 0 || g->mtide > xm::MT_MAX || (g->mtide > 0 && !g->tcp)) {
    set_error("efdc_xm_create: member %d: MTIDE must be in 0..%d with TCP given", mi, xm::MT_MAX);
    return false;
  }
  int imin = INT32_MAX, imax = INT32_MIN, jmin = INT32_MAX, jmax = INT32_MIN;
  for (int L = 2; L <= la; ++L) {
    imin = std::min(imin, g->il[L - 1]);
    imax = std::max(imax, g->il[L - 1]);
    jmin = std::min(jmin, g->jl[L - 1]);
    jmax = std::max(jmax, g->jl[L - 1]);
  }
  const long ni = long(imax) - imin + 1, nj = long(jmax) - jmin + 1;
  if (ni <= 0 || nj <= 0 || ni * nj > (1L << 31) - 1) {
    set_error("efdc_xm_create: member %d: bad IL/JL range", mi);
    return false;
  }
  std::vector<int> lij(size_t(ni * nj), 0);
  for (int L = 2; L <= la; ++L) {
    const long k = long(g->jl[L - 1] - jmin) * ni + (g->il[L - 1] - imin);
    if (lij[k]) {
      set_error("efdc_xm_create: member %d: cells %d and %d share (I,J)", mi, lij[k], L);
      return false;
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
      set_error("efdc_xm_create: member %d, cell L=%d (I=%d,J=%d): LNC/LSC/LEC/LWC are not the "
                "maps of a structured grid (periodic ISCONNECT links are not supported)",
                mi, L, i, j);
      return false;
    }
  }
  ml.imin = imin;
  ml.jmin = jmin;
  ml.ntx = int((ni + xm::TX - 1) / xm::TX);
  ml.nty = int((nj + xm::TY - 1) / xm::TY);
  ml.tile_of.assign(size_t(ml.ntx) * ml.nty, 0);
  for (int L = 2; L <= la; ++L) {
    const int tx = (g->il[L - 1] - imin) / xm::TX, ty = (g->jl[L - 1] - jmin) / xm::TY;
    int &t = ml.tile_of[size_t(ty) * ml.ntx + tx];
    if (!t) {
      t = -1;
      ml.tiles.push_back({morton2(tx, ty), ty * ml.ntx + tx});
    }
  }
  std::sort(ml.tiles.begin(), ml.tiles.end());
  for (size_t k = 0; k < ml.tiles.size(); ++k) ml.tile_of[ml.tiles[k].second] = int(k) + 1;
  return true;
}

// The status of a batch call: the first member error, else NEG_DEPTH if any
// member had one, else OK.
int overall_status(const efdc_xm_stats *st, int M) {
  int worst = EFDC_XM_OK;
  for (int m = 0; m < M; ++m) {
    const int s = st[m].status;
    if (s == EFDC_XM_OK) continue;
    if (s == EFDC_XM_NEG_DEPTH) {
      if (worst == EFDC_XM_OK) worst = s;
      continue;
    }
    if (worst == EFDC_XM_OK || worst == EFDC_XM_NEG_DEPTH) worst = s;
  }
  return worst;
}

void fill_status(efdc_xm_stats *st, int M, int status) {
  for (int m = 0; m < M; ++m) st[m].status = status;
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
  if (c->mom_lists) cudaFree(c->mom_lists);
  if (c->pack_h) cudaFreeHost(c->pack_h);
  void *pinned[] = {c->ctl_h, c->glob_h, c->act_h, c->mpoly_h, c->sc_h, c->jobs_h, c->pser_h};
  for (void *p : pinned)
    if (p) cudaFreeHost(p);
  if (c->gslot) cudaFree(c->gslot);
  if (c->gbuf) cudaFree(c->gbuf);
  for (cudaGraphExec_t g : c->graph_cg)
    if (g) cudaGraphExecDestroy(g);
  for (cudaGraphExec_t g : c->graph_mx)
    if (g) cudaGraphExecDestroy(g);
  for (StepGraph &g : c->step_graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (cudaStream_t s : c->cap_stream)
    if (s) cudaStreamDestroy(s);
  for (void *b : c->chan_bufs) cudaFree(b);
  for (cudaStream_t s : c->copy_stream)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : c->copy_event)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t s : c->dn_stream)
    if (s) cudaStreamDestroy(s);
  for (cudaStream_t s : {c->up_x, c->dn_x})
    if (s) cudaStreamDestroy(s);
  for (int k = 0; k < NCHUNK; ++k) {
    for (cudaEvent_t e : {c->ev_up[k], c->ev_step[k], c->ev_g[k]})
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : c->ev_j[k])
      if (e) cudaEventDestroy(e);
  }
  if (c->ev_start) cudaEventDestroy(c->ev_start);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int32_t efdc_xm_nmembers(const efdc_xm_ctx *c) { return c ? c->M : 0; }

efdc_xm_ctx *efdc_xm_create_batch(const efdc_xm_grid *grids, int32_t nmembers, int32_t device) {
  g_last_error.clear();
  if (!grids || nmembers < 1) {
    set_error("efdc_xm_create: need a grid for each of nmembers >= 1 members");
    return nullptr;
  }
  const int M = nmembers;
  std::vector<MemberLayout> ml(M);
  long long nt = 1;
  for (int m = 0; m < M; ++m) {
    if (!member_layout(&grids[m], m, ml[m])) return nullptr;
    nt += (long long)ml[m].tiles.size();
  }
  if (nt * TILE > (long long)INT32_MAX) {
    set_error("efdc_xm_create: %lld tiles exceed the 32-bit slot index", nt);
    return nullptr;
  }

  efdc_xm_ctx *c = new efdc_xm_ctx();
  c->device = device;
  c->M = M;
  c->mem.resize(M);
  // each member: its ghost tile (all land slots, holding the member's own
  // ghost cell LC), then its water tiles; tile 0 is member 0's ghost tile
  int ntile = 0;
  long long off = 0;
  for (int m = 0; m < M; ++m) {
    Member &mb = c->mem[m];
    mb.la = grids[m].la;
    mb.lc = grids[m].lc;
    ntile += 1;
    mb.tile0 = ntile;
    ntile += int(ml[m].tiles.size());
    mb.tile1 = ntile;
    mb.off = off;
    off += mb.lc + 1;
    mb.mtide = grids[m].mtide;
    if (mb.mtide > 0) mb.tcp.assign(grids[m].tcp, grids[m].tcp + mb.mtide);
  }
  c->ntile = ntile;
  c->nslot = ntile * TILE;
  c->stage_len = off;
  for (const Member &mb : c->mem)  // the member windows of k_cg_small
    c->small_slots = std::max(c->small_slots, (mb.tile1 - mb.tile0 + 1) * TILE);
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
  for (cudaStream_t &s : c->copy_stream)
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
      return bail("stream creation failed");
  for (cudaEvent_t &e : c->copy_event)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      return bail("event creation failed");
  {
    bool ok = cudaStreamCreateWithFlags(&c->up_x, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&c->dn_x, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->ev_start, cudaEventDisableTiming) == cudaSuccess;
    for (cudaStream_t &s : c->dn_stream)
      ok = ok && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    for (int k = 0; k < NCHUNK; ++k) {
      for (cudaEvent_t *e : {&c->ev_up[k], &c->ev_step[k], &c->ev_g[k]})
        ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
      for (cudaEvent_t &e : c->ev_j[k])
        ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
    }
    if (!ok) return bail("stream or event creation failed");
  }
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);

  // ---- host layout: tiles, quads (4-tile CG units, never across members), slots ----
  std::vector<int4> tnbr(ntile, int4{0, 0, 0, 0});
  std::vector<int> tile_member(ntile, 0), tend(M), qstart(M + 1, 0);
  std::vector<int4> quads;
  std::vector<uint8_t> kind(c->nslot, xm::LAND);
  std::vector<int> lidx(c->nslot, 0);
  std::vector<std::vector<int>> slot_of(M);
  for (int m = 0; m < M; ++m) {
    const efdc_xm_grid *g = &grids[m];
    const MemberLayout &ly = ml[m];
    Member &mb = c->mem[m];
    for (size_t k = 0; k < ly.tiles.size(); ++k) {
      const int id = ly.tiles[k].second, tx = id % ly.ntx, ty = id / ly.ntx;
      const int ghost = mb.tile0 - 1;  // a missing neighbour tile: the member's ghost
      auto tl = [&](int x, int y) {
        if (x < 0 || y < 0 || x >= ly.ntx || y >= ly.nty) return ghost;
        const int t = ly.tile_of[size_t(y) * ly.ntx + x];
        return t > 0 ? mb.tile0 + t - 1 : ghost;
      };
      const int gt = mb.tile0 + int(k);
      tnbr[gt] = int4{tl(tx - 1, ty), tl(tx + 1, ty), tl(tx, ty - 1), tl(tx, ty + 1)};
      tile_member[gt] = m;
    }
    tnbr[mb.tile0 - 1] = int4{mb.tile0 - 1, mb.tile0 - 1, mb.tile0 - 1, mb.tile0 - 1};
    tile_member[mb.tile0 - 1] = m;
    tend[m] = mb.tile1;
    qstart[m] = int(quads.size());
    for (int t = mb.tile0; t < mb.tile1; t += 4)
      quads.push_back(int4{m, t, std::min(4, mb.tile1 - t), 0});
    qstart[m + 1] = int(quads.size());
    slot_of[m].assign(size_t(mb.lc) + 1, 0);
    for (int L = 2; L <= mb.la; ++L) {
      const int ii = g->il[L - 1] - ly.imin, jj = g->jl[L - 1] - ly.jmin;
      const int t = ly.tile_of[size_t(jj / xm::TY) * ly.ntx + ii / xm::TX];
      const int d = (mb.tile0 + t - 1) * TILE + (jj % xm::TY) * xm::TX + (ii % xm::TX);
      kind[d] = xm::WATER;
      lidx[d] = L;
      slot_of[m][L] = d;
    }
  }
  c->nquad = int(quads.size());

  // ---- open boundaries, packed per member in the W, E, S, N loop order ----
  int mtmax = 1;
  for (int m = 0; m < M; ++m) mtmax = std::max(mtmax, grids[m].mtide);
  std::vector<int> bslot, bnbr, bside, bispb, bmember, bstart(M + 1, 0), bmt(M);
  std::vector<double> bpcb, bpsb;
  for (int m = 0; m < M; ++m) {
    const efdc_xm_grid *g = &grids[m];
    Member &mb = c->mem[m];
    mb.b0 = int(bslot.size());
    bstart[m] = mb.b0;
    bmt[m] = g->mtide;
    std::unordered_set<int> bcells, targets;
    for (int s = 0; s < 4; ++s) {
      const efdc_xm_obc &o = g->obc[s];
      if (o.n < 0 || (o.n > 0 && (!o.l || !o.ispb))) return bail("bad open-boundary arrays");
      for (int ll = 0; ll < o.n; ++ll) bcells.insert(o.l[ll]);
    }
    for (int s = 0; s < 4; ++s) {
      const efdc_xm_obc &o = g->obc[s];
      mb.side_n[s] = o.n;
      for (int ll = 0; ll < o.n; ++ll) {
        const int L = o.l[ll];
        if (L < 2 || L > mb.la) return bail("open-boundary L out of range");
        const int nbL = (s == 0) ? g->lec[L - 1] : (s == 1) ? g->lwc[L - 1]
                        : (s == 2) ? g->lnc[L - 1] : g->lsc[L - 1];
        bslot.push_back(slot_of[m][L]);
        // the ghost cell LC: a slot of the member's ghost tile
        bnbr.push_back(nbL == mb.lc ? (mb.tile0 - 1) * TILE : slot_of[m][nbL]);
        bside.push_back(s);
        bispb.push_back(o.ispb[ll]);
        bmember.push_back(m);
        for (int t = 0; t < mtmax; ++t) {
          const bool have = t < g->mtide;
          bpcb.push_back(have && o.pcb ? o.pcb[size_t(t) * o.ld + ll] : 0.0);
          bpsb.push_back(have && o.psb ? o.psb[size_t(t) * o.ld + ll] : 0.0);
        }
        kind[slot_of[m][L]] = xm::OPENBC;
        if (o.ispb[ll] == 1 || o.ispb[ll] == 2) mb.may_asym = true;
        if (o.ispb[ll] == 2) {
          // W: the cell after L in the numbering; S: L's north neighbour
          const int Lm = s == 0 ? L + 1 : s == 2 ? g->lnc[L - 1] : L;
          if (Lm >= 2 && Lm <= mb.la) {
            const int nb2 = s == 0 ? g->lnc[Lm - 1] : s == 1 ? g->lwc[Lm - 1]
                            : s == 2 ? g->lec[Lm - 1] : g->lsc[Lm - 1];
            mb.t2.push_back(int4{s, Lm, nb2, 0});
          }
        }
        // hazard: a ghost or boundary-cell target, or a target shared by two
        // boundary cells, needs the reference's serial loop order
        if (nbL == mb.lc || bcells.count(nbL) || !targets.insert(nbL).second) c->obc_serial = true;
      }
    }
    mb.nobc = int(bslot.size()) - mb.b0;
    c->any_may_asym |= mb.may_asym;
  }
  bstart[M] = int(bslot.size());
  c->nobc = int(bslot.size());

  // ---- launch geometry ----
  const int occ = xm::occupancy_blocks_per_sm();
  c->grid = std::max(1, std::min(c->ntile - 1, c->nsm * occ));
  auto qgrid = [&](int per_sm) { return std::max(1, std::min(c->nquad, c->nsm * per_sm)); };
  c->grid_cg = qgrid(xm::occupancy_blocks_per_sm_cg());
  c->grid_cg32 = qgrid(xm::occupancy_blocks_per_sm_mixed());
  c->grid_up32 = qgrid(xm::occupancy_blocks_per_sm_mixed_update());

  // ---- device arrays ----
  const size_t ns = c->nslot;
  c->lidx = c->alloc<int>(ns);
  c->tile_member = c->alloc<int>(ntile);
  int4 *tnbr_d = c->alloc<int4>(ntile);
  uint8_t *kind_d = c->alloc<uint8_t>(ns);
  int4 *quads_d = c->alloc<int4>(quads.size());
  int *qstart_d = c->alloc<int>(M + 1), *tend_d = c->alloc<int>(M);
  c->moff = c->alloc<long long>(M);
  c->mlc = c->alloc<int>(M);
  c->sc = c->alloc<xm::StepScalars>(M);
  c->ctl = c->alloc<Ctl>(M);
  c->glob = c->alloc<Glob>(1);
  c->act = c->alloc<int>(M);
  c->mpoly = c->alloc<int>(M);
  c->part = c->alloc<double>(2 * size_t(c->nquad) + 64);
  if (!c->lidx || !c->tile_member || !tnbr_d || !kind_d || !quads_d || !qstart_d || !tend_d ||
      !c->moff || !c->mlc || !c->sc || !c->ctl || !c->glob || !c->act || !c->mpoly || !c->part)
    return bail("cudaMalloc failed");
  {
    std::vector<long long> moff(M);
    std::vector<int> mlc(M);
    for (int m = 0; m < M; ++m) {
      moff[m] = c->mem[m].off;
      mlc[m] = c->mem[m].lc;
    }
    cudaMemcpy(c->moff, moff.data(), M * sizeof(long long), cudaMemcpyHostToDevice);
    cudaMemcpy(c->mlc, mlc.data(), M * sizeof(int), cudaMemcpyHostToDevice);
  }
  cudaMemcpy(c->lidx, lidx.data(), ns * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(c->tile_member, tile_member.data(), ntile * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(tnbr_d, tnbr.data(), tnbr.size() * sizeof(int4), cudaMemcpyHostToDevice);
  cudaMemcpy(kind_d, kind.data(), ns, cudaMemcpyHostToDevice);
  c->kind_h = kind;
  c->chans.assign(M, {});
  c->hp1_h.assign(M, 1.0);
  c->chan_start.assign(M + 1, 0);
  c->qstart_h = qstart;
  for (int m = 0; m < M; ++m) c->small_units = std::max(c->small_units, qstart[m + 1] - qstart[m]);
  c->has_layers.assign(M, 0);
  cudaMemcpy(quads_d, quads.data(), quads.size() * sizeof(int4), cudaMemcpyHostToDevice);
  cudaMemcpy(qstart_d, qstart.data(), (M + 1) * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(tend_d, tend.data(), M * sizeof(int), cudaMemcpyHostToDevice);
  auto D = [&]() { return c->alloc<double>(ns); };
  auto I = [&]() { return c->alloc<int>(ns); };
  auto Fl = [&]() { return c->alloc<float>(ns); };
  xm::DevStatic &S = c->S;
  S.tnbr = tnbr_d;
  S.kind = kind_d;
  S.lidx = c->lidx;
  S.tile_member = c->tile_member;
  S.quads = quads_d;
  S.qstart = qstart_d;
  S.tend = tend_d;
  S.sc = c->sc;
  S.nquad = c->nquad;
  S.nmember = M;
  double *st[18];
  for (double *&p : st) p = D();
  S.dxyp = st[0]; S.dxyip = st[1]; S.dxiu = st[2]; S.dyiu = st[3]; S.dxiv = st[4];
  S.dyiv = st[5]; S.dxyu = st[6]; S.dxyv = st[7]; S.hruo = st[8]; S.hrvo = st[9];
  S.subo = st[10]; S.svbo = st[11]; S.sbxo = st[12]; S.sbyo = st[13]; S.belv = st[14];
  S.fsgzu = st[16]; S.fsgzv = st[17];
  xm::DevState &X = c->X;
  X.rcx = st[15];
  X.rcy = D();
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
  // the views of a CALPUV2C step (reset by every step after its swaps)
  X.huc = X.hu; X.hvc = X.hv; X.hb = X.h1p; X.ub = X.uhdy1e; X.vb = X.vhdx1e; X.hp0 = X.h1p;
  xm::DevSystem &Y = c->Y;
  Y.ccc = D(); Y.ccs = D(); Y.ccw = D(); Y.cce = D(); Y.ccn = D(); Y.fptmp = D();
  Y.r = D(); Y.pa = D(); Y.pb = D(); Y.ap = D(); Y.z = D();
  Y.as32 = Fl(); Y.aw32 = Fl(); Y.ae32 = Fl(); Y.an32 = Fl();
  Y.r32 = Fl(); Y.pa32 = Fl(); Y.pb32 = Fl(); Y.ap32 = Fl(); Y.x32 = Fl(); Y.z32 = Fl();
  Y.r32b = Fl();
  Y.mpoly = c->mpoly;
  Y.err = c->glob ? &c->glob->err : nullptr;
  c->ptmp = D();
  c->mxview = xm::SysView{X.fp, X.cc, X.cs, X.cw, X.ce, X.cn, 1};
  if (!c->ptmp || !Y.x32 || !Y.z32 || !Y.r32b || !X.rcy)
    return bail("cudaMalloc failed (device memory)");
  auto pin = [](void *pp, size_t bytes) {
    return cudaHostAlloc(static_cast<void **>(pp), std::max<size_t>(bytes, 1),
                         cudaHostAllocMapped) == cudaSuccess;
  };
  if (!pin(&c->ctl_h, sizeof(Ctl) * M) || !pin(&c->glob_h, sizeof(Glob)) ||
      !pin(&c->act_h, sizeof(int) * M) || !pin(&c->mpoly_h, sizeof(int) * M) ||
      !pin(&c->sc_h, sizeof(xm::StepScalars) * M) ||
      !pin(&c->jobs_h, sizeof(CopyJob) * MAX_JOBS))
    return bail("cudaHostAlloc failed");
  std::memset(c->ctl_h, 0, sizeof(Ctl) * M);
  std::memset(c->sc_h, 0, sizeof(xm::StepScalars) * M);
  {  // the control mirrors' device addresses (pinned memory is mapped under UVA)
    void *h[] = {c->ctl_h, c->glob_h, c->act_h, c->mpoly_h, c->sc_h};
    void **d[] = {&c->ctl_hd, &c->glob_hd, &c->act_hd, &c->mpoly_hd, &c->sc_hd};
    bool ok = true;
    for (int k = 0; k < 5; ++k) ok = ok && cudaHostGetDevicePointer(d[k], h[k], 0) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      for (void **p : d) *p = nullptr;
    }
  }
  c->jobs_d = c->alloc<CopyJob>(MAX_JOBS);
  if (!c->jobs_d) return bail("cudaMalloc failed");
  {  // land slots of the scaled system: CCC=1 keeps them inert in the CG;
     // RCX/RCY = 1 on water cells, 0 on the ghosts (calpuv2c.f90:97-102)
    std::vector<double> one(ns, 0.0), rc(ns, 0.0), fu(ns, 1.0), fv(ns, 1.0);
    for (size_t d = 0; d < ns; ++d)
      if (kind[d] == xm::LAND) one[d] = 1.0;
    for (int m = 0; m < M; ++m)
      for (int L = 2; L <= c->mem[m].la; ++L) {
        const int d = slot_of[m][L];
        rc[d] = 1.0;
        fu[d] = 0.5 / grids[m].dxyu[L - 1];  // calpuv2c.f90:111-116
        fv[d] = 0.5 / grids[m].dxyv[L - 1];
      }
    cudaMemcpy(Y.ccc, one.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(X.rcx, rc.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(X.rcy, rc.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(st[16], fu.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(st[17], fv.data(), ns * sizeof(double), cudaMemcpyHostToDevice);
  }
  for (int k = 0; k < NSTAGE; ++k) {
    double *p = c->alloc<double>(size_t(c->stage_len), false);
    if (!p) return bail("cudaMalloc failed (staging)");
    c->stage.push_back(p);
  }
  xm::DevObc &Bo = c->B;
  Bo.n = c->nobc;
  Bo.mtmax = mtmax;
  {
    int *bmt_d = c->alloc<int>(M), *bstart_d = c->alloc<int>(M + 1);
    if (!bmt_d || !bstart_d) return bail("cudaMalloc failed (obc)");
    cudaMemcpy(bmt_d, bmt.data(), M * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(bstart_d, bstart.data(), (M + 1) * sizeof(int), cudaMemcpyHostToDevice);
    Bo.mtide = bmt_d;
    Bo.bstart = bstart_d;
  }
  if (c->nobc > 0) {
    const int n = c->nobc;
    int *bs = c->alloc<int>(n), *bn = c->alloc<int>(n), *bd = c->alloc<int>(n),
        *bi = c->alloc<int>(n), *bm = c->alloc<int>(n);
    double *pc = c->alloc<double>(bpcb.size()), *ps = c->alloc<double>(bpsb.size());
    c->pser_d = c->alloc<double>(n);
    if (!bs || !bn || !bd || !bi || !bm || !pc || !ps || !c->pser_d)
      return bail("cudaMalloc failed (obc)");
    cudaMemcpy(bs, bslot.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(bn, bnbr.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(bd, bside.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(bi, bispb.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(bm, bmember.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(pc, bpcb.data(), bpcb.size() * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(ps, bpsb.data(), bpsb.size() * sizeof(double), cudaMemcpyHostToDevice);
    Bo.slot = bs;
    Bo.nbr = bn;
    Bo.side = bd;
    Bo.ispb = bi;
    Bo.member = bm;
    Bo.pcb = pc;
    Bo.psb = ps;
    Bo.pser = c->pser_d;
    if (!pin(&c->pser_h, n * sizeof(double))) return bail("cudaHostAlloc failed");
  }
  // the zero-fills above ran on the legacy stream; finish them before any
  // work on the non-blocking solver stream
  if (cudaDeviceSynchronize() != cudaSuccess) return bail("device error during allocation");
  // static metrics into tile order (land slots take element LC of their member)
  auto per = [&](const double *efdc_xm_grid::*f) {
    std::vector<const void *> v(M);
    for (int m = 0; m < M; ++m) v[m] = grids[m].*f;
    return v;
  };
  const std::pair<const double *efdc_xm_grid::*, double *> metrics[] = {
      {&efdc_xm_grid::dxyp, st[0]},   {&efdc_xm_grid::dxyip, st[1]}, {&efdc_xm_grid::dxiu, st[2]},
      {&efdc_xm_grid::dyiu, st[3]},   {&efdc_xm_grid::dxiv, st[4]},  {&efdc_xm_grid::dyiv, st[5]},
      {&efdc_xm_grid::dxyu, st[6]},   {&efdc_xm_grid::dxyv, st[7]},  {&efdc_xm_grid::hruo, st[8]},
      {&efdc_xm_grid::hrvo, st[9]},   {&efdc_xm_grid::subo, st[10]}, {&efdc_xm_grid::svbo, st[11]},
      {&efdc_xm_grid::sbxo, st[12]},  {&efdc_xm_grid::sbyo, st[13]}, {&efdc_xm_grid::belv, st[14]}};
  std::vector<Xfer> xs;
  for (const auto &mt : metrics) xs.push_back(Xfer{per(mt.first), mt.second, 0});
  if (upload_arrays(c, xs) != EFDC_XM_OK) return bail("upload of the static arrays failed");
  if (cudaDeviceSynchronize() != cudaSuccess) return bail("device error during set-up");
  for (int m = 0; m < M; ++m) c->mem[m].slot_of = std::move(slot_of[m]);
  return c;
}

efdc_xm_ctx *efdc_xm_create(const efdc_xm_grid *g, int32_t device) {
  if (!g) {
    g_last_error.clear();
    set_error("efdc_xm_create: grid is NULL");
    return nullptr;
  }
  return efdc_xm_create_batch(g, 1, device);
}

namespace {
int upload_batch(efdc_xm_ctx *c, const efdc_xm_fields *f, bool skip_wetdry, bool skip_sbxy,
                 bool levels);
}

int32_t efdc_xm_upload_batch(efdc_xm_ctx *c, const efdc_xm_fields *f) {
  return upload_batch(c, f, false, false, f && f[0].p1);
}

namespace {
// The buffers of the three time levels, on first use.
int ensure_levels(efdc_xm_ctx *c) {
  if (c->tl3_alloc) return EFDC_XM_OK;
  xm::DevState &X = c->X;
  double *b[14];
  for (double *&p : b) {
    p = c->alloc<double>(size_t(c->nslot));  // zeroed: HUTMP, HVTMP stay 0 on land slots
    if (!p) {
      set_error("cudaMalloc failed (device memory for the three time levels)");
      return EFDC_XM_CUDA_ERROR;
    }
  }
  X.p1 = b[0]; X.h2p = b[1]; X.uhdy2e = b[2]; X.vhdx2e = b[3]; X.h1u = b[4]; X.h1v = b[5];
  X.hutmp = b[6]; X.hvtmp = b[7]; X.fpgxe = b[8]; X.fpgye = b[9];
  X.tsx1 = b[10]; X.tsy1 = b[11]; X.tbx1 = b[12]; X.tby1 = b[13];
  CK(cudaDeviceSynchronize());  // the zeroing ran on the legacy stream
  c->tl3_alloc = true;
  return EFDC_XM_OK;
}

// The views of the step about to run (DevState::huc ... hp0), after its
// time-level swaps.
void set_views(efdc_xm_ctx *c, int istl) {
  xm::DevState &X = c->X;
  const bool corr = istl == 2, leap = istl == 3;
  X.huc = corr ? X.hutmp : X.hu;
  X.hvc = corr ? X.hvtmp : X.hv;
  X.hb = leap ? X.h2p : X.h1p;
  X.ub = leap ? X.uhdy2e : X.uhdy1e;
  X.vb = leap ? X.vhdx2e : X.vhdx1e;
  X.hp0 = corr ? X.hp : X.h1p;
}
}  // namespace

namespace {
// skip_wetdry: leave out the fields that only wetting and drying reads
// (LMASKDRY, ISCDRY, NATDRY, QDWASTE, VDWASTE), for a step in which no member
// has it; skip_sbxy: SBX, SBY as well (read also by the baroclinic terms).
// Their device copies are then marked out of date.  levels: upload the three
// time levels of CALPUV9C (P1, H2P, H1P, UHDY1E ... FPGYE) as well.
// The arrays of an upload, with its argument checks.
// The implicit drag's input arrays, allocated (zeroed: FXVEGE = FYVEGE = 0
// unless given) by the first upload that carries one of them.
int ensure_drag(efdc_xm_ctx *c) {
  if (c->drag_alloc) return EFDC_XM_OK;
  xm::DevState &X = c->X;
  const double **a[] = {&X.ubot, &X.vbot, &X.vu, &X.uv, &X.stbx, &X.stby, &X.fxvege, &X.fyvege};
  for (const double **p : a) {
    double *d = c->alloc<double>(size_t(c->nslot));
    if (!d) {
      set_error("cudaMalloc failed (implicit drag inputs)");
      return EFDC_XM_CUDA_ERROR;
    }
    *p = d;
  }
  c->drag_alloc = true;
  return EFDC_XM_OK;
}

// Bits of ctx::drag_in: the implicit drag inputs the device holds.
enum : unsigned { DRAG_BED = 1u, DRAG_VEG = 2u };

// Arrays written by a step without wetting and drying, and by any step
// (their device copies stop matching the caller's).
constexpr uint32_t STEP_WRITES_DRYFREE = EFDC_XM_SAME_P | EFDC_XM_SAME_HP | EFDC_XM_SAME_HU |
                                         EFDC_XM_SAME_HV | EFDC_XM_SAME_UHDYE |
                                         EFDC_XM_SAME_VHDXE | EFDC_XM_SAME_LOPENBCDRY;
constexpr uint32_t STEP_WRITES =
    EFDC_XM_SAME_P | EFDC_XM_SAME_HP | EFDC_XM_SAME_HU | EFDC_XM_SAME_HV | EFDC_XM_SAME_UHDYE |
    EFDC_XM_SAME_VHDXE | EFDC_XM_SAME_SUB | EFDC_XM_SAME_SVB | EFDC_XM_SAME_SBX |
    EFDC_XM_SAME_SBY | EFDC_XM_SAME_LMASKDRY | EFDC_XM_SAME_ISCDRY | EFDC_XM_SAME_LOPENBCDRY |
    EFDC_XM_SAME_NATDRY | EFDC_XM_SAME_QDWASTE | EFDC_XM_SAME_VDWASTE;

// The arrays of an upload.  An array whose bit the caller set in `unchanged`
// and whose device copy is still its last transfer is left out; *sent gets
// the bits of the arrays that go.
int plan_upload(efdc_xm_ctx *c, const efdc_xm_fields *f, bool skip_wetdry, bool skip_sbxy,
                bool levels, std::vector<Xfer> &xs, uint32_t *sent = nullptr) {
  xm::DevState &X = c->X;
  const int M = c->M;
  for (int m = 1; m < M; ++m)
    if (f[m].unchanged != f[0].unchanged) {
      set_error("efdc_xm_upload: member %d: the unchanged bits differ from member 0's", m);
      return EFDC_XM_BAD_ARGUMENT;
    }
  const uint32_t skip = f[0].unchanged & c->synced;
  uint32_t went = 0;
  for (int m = 0; m < M; ++m)
    if (!c->chans[m].empty() && (!f[m].qchanu || !f[m].qchanv || !f[m].qchanun || !f[m].qchanvn)) {
      set_error("efdc_xm_upload: member %d has sub-grid channels: QCHANU, QCHANV, QCHANUN and "
                "QCHANVN are required", m);
      return EFDC_XM_BAD_ARGUMENT;
    }
  int rc = 0;
#define XM_UP(name, dev, kind)                                   \
  {                                                              \
    std::vector<const void *> v(M);                              \
    for (int m = 0; m < M; ++m) v[m] = f[m].name;                \
    if ((rc = collect(c, xs, v, dev, kind, #name))) return rc;   \
  }
#define XM_UPB(name, dev, kind, bit)                             \
  if (!(skip & (bit))) {                                         \
    const size_t n0 = xs.size();                                 \
    XM_UP(name, dev, kind)                                       \
    if (xs.size() > n0) went |= (bit);                           \
  }
  XM_UPB(p, X.p, 0, EFDC_XM_SAME_P) XM_UPB(hp, X.hp, 0, EFDC_XM_SAME_HP)
  XM_UPB(hu, X.hu, 0, EFDC_XM_SAME_HU) XM_UPB(hv, X.hv, 0, EFDC_XM_SAME_HV)
  XM_UPB(uhdye, X.uhdye, 0, EFDC_XM_SAME_UHDYE) XM_UPB(vhdxe, X.vhdxe, 0, EFDC_XM_SAME_VHDXE)
  XM_UPB(sub, X.sub, 0, EFDC_XM_SAME_SUB) XM_UPB(svb, X.svb, 0, EFDC_XM_SAME_SVB)
  XM_UPB(lopenbcdry, X.lopenbcdry, 1, EFDC_XM_SAME_LOPENBCDRY)
  XM_UPB(fcaxe, X.fcaxe, 0, EFDC_XM_SAME_FCAXE) XM_UPB(fcaye, X.fcaye, 0, EFDC_XM_SAME_FCAYE)
  XM_UPB(fxe, X.fxe, 0, EFDC_XM_SAME_FXE) XM_UPB(fye, X.fye, 0, EFDC_XM_SAME_FYE)
  XM_UPB(tsx, X.tsx, 0, EFDC_XM_SAME_TSX) XM_UPB(tsy, X.tsy, 0, EFDC_XM_SAME_TSY)
  XM_UPB(tbx, X.tbx, 0, EFDC_XM_SAME_TBX) XM_UPB(tby, X.tby, 0, EFDC_XM_SAME_TBY)
  XM_UPB(qsume, X.qsume, 0, EFDC_XM_SAME_QSUME)
  if (!skip_sbxy) {
    XM_UPB(sbx, X.sbx, 0, EFDC_XM_SAME_SBX) XM_UPB(sby, X.sby, 0, EFDC_XM_SAME_SBY)
  }
  if (!skip_wetdry) {
    XM_UPB(lmaskdry, X.lmaskdry, 1, EFDC_XM_SAME_LMASKDRY)
    XM_UPB(iscdry, X.iscdry, 2, EFDC_XM_SAME_ISCDRY)
    XM_UPB(natdry, X.natdry, 2, EFDC_XM_SAME_NATDRY)
    XM_UPB(qdwaste, X.qdwaste, 0, EFDC_XM_SAME_QDWASTE)
    XM_UPB(vdwaste, X.vdwaste, 0, EFDC_XM_SAME_VDWASTE)
  }
  {  // the implicit drag's inputs; UHE, VHE go with them (read at entry)
    bool any = false;
    for (int m = 0; m < M && !any; ++m)
      any = f[m].ubot || f[m].vbot || f[m].vu || f[m].uv || f[m].stbx || f[m].stby ||
            f[m].fxvege || f[m].fyvege;
    if (any) {
      if ((rc = ensure_drag(c))) return rc;
      XM_UP(ubot, X.ubot, 0) XM_UP(vbot, X.vbot, 0) XM_UP(vu, X.vu, 0) XM_UP(uv, X.uv, 0)
      XM_UP(stbx, X.stbx, 0) XM_UP(stby, X.stby, 0) XM_UP(fxvege, X.fxvege, 0)
      XM_UP(fyvege, X.fyvege, 0) XM_UP(uhe, X.uhe, 0) XM_UP(vhe, X.vhe, 0)
    }
  }
  if (sent) *sent = went;
#undef XM_UPB
  if (levels) {
    for (int m = 0; m < M; ++m) {
      const efdc_xm_fields &x = f[m];
      if (!x.p1 || !x.h2p || !x.h1p || !x.uhdy1e || !x.vhdx1e || !x.uhdy2e || !x.vhdx2e ||
          !x.h1u || !x.h1v) {
        set_error("member %d: the three time levels need P1, H2P, H1P, UHDY1E, VHDX1E, UHDY2E, "
                  "VHDX2E, H1U and H1V", m);
        return EFDC_XM_BAD_ARGUMENT;
      }
    }
    if ((rc = ensure_levels(c))) return rc;
    XM_UP(p1, X.p1, 0) XM_UP(h2p, X.h2p, 0) XM_UP(h1p, X.h1p, 0)
    XM_UP(uhdy1e, X.uhdy1e, 0) XM_UP(vhdx1e, X.vhdx1e, 0)
    XM_UP(uhdy2e, X.uhdy2e, 0) XM_UP(vhdx2e, X.vhdx2e, 0)
    XM_UP(h1u, X.h1u, 0) XM_UP(h1v, X.h1v, 0)
    XM_UP(tsx1, X.tsx1, 0) XM_UP(tsy1, X.tsy1, 0) XM_UP(tbx1, X.tbx1, 0) XM_UP(tby1, X.tby1, 0)
    XM_UP(fpgxe, X.fpgxe, 0) XM_UP(fpgye, X.fpgye, 0)
  }
#undef XM_UP
  // B(L,K), one staging job per layer; a member without B gets zeros
  bool anyb = false;
  for (int m = 0; m < M; ++m) anyb |= f[m].b != nullptr;
  if (anyb && c->S.baro.kc > 0) {
    for (int m = 0; m < M; ++m)
      if (f[m].b && f[m].b_ld < c->mem[m].lc) {
        set_error("efdc_xm_upload: member %d: b_ld %d < LC", m, f[m].b_ld);
        return EFDC_XM_BAD_ARGUMENT;
      }
    for (int k = 0; k < c->S.baro.kc; ++k) {
      std::vector<const void *> v(M);
      for (int m = 0; m < M; ++m)
        v[m] = f[m].b ? static_cast<const void *>(f[m].b + size_t(k) * f[m].b_ld)
                      : static_cast<const void *>(c->zeros_h.data());
      xs.push_back(Xfer{v, c->S.baro.b + size_t(k) * c->S.baro.stride, 0});
    }
  }
  return EFDC_XM_OK;
}

// Two time levels: the second buffer of each time-level pair starts as a copy
// of the slots [d0, d1) (its land slots must hold the ghost values too; the
// H1P input is not used because a CALPUV2C step begins with H1P = HP,
// calpuv2c.f90:264).
// Copied by a kernel (no copy engine: see to_device).
int copy_levels(efdc_xm_ctx *c, const efdc_xm_fields *f, size_t d0, size_t d1, cudaStream_t st) {
  const xm::DevState &X = c->X;
  const size_t nb = (d1 - d0) * sizeof(double);
  if (f[0].uhdye) xm::launch_words(st, X.uhdy1e + d0, X.uhdye + d0, nb);
  if (f[0].vhdxe) xm::launch_words(st, X.vhdx1e + d0, X.vhdxe + d0, nb);
  if (f[0].hp) xm::launch_words(st, X.h1p + d0, X.hp + d0, nb);
  CK(cudaGetLastError());
  return EFDC_XM_OK;
}

// The small per-member uploads: open-boundary series, channel flows, HP(1).
// Waits for them (and for the solver stream's earlier work).
int upload_small(efdc_xm_ctx *c, const efdc_xm_fields *f) {
  const int M = c->M;
  if (c->nobc > 0) {
    for (int m = 0; m < M; ++m) {
      int k = c->mem[m].b0;
      for (int s = 0; s < 4; ++s)
        for (int ll = 0; ll < c->mem[m].side_n[s]; ++ll, ++k)
          c->pser_h[k] = f[m].pser[s] ? f[m].pser[s][ll] : 0.0;
    }
    CK(cudaMemcpyAsync(c->pser_d, c->pser_h, c->nobc * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
  }
  if (c->S.ch.n > 0) {  // the channels' flows and HP(1) (subchan.f90:84)
    const xm::DevChan &C = c->S.ch;
    for (int m = 0; m < M; ++m) {
      const int k0 = c->chan_start[m], n = c->chan_start[m + 1] - k0;
      if (f[m].hp) c->hp1_h[m] = f[m].hp[0];
      if (n == 0) continue;
      const size_t b = sizeof(double) * size_t(n);
      CK(cudaMemcpyAsync(C.qu + k0, f[m].qchanu, b, cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemcpyAsync(C.qv + k0, f[m].qchanv, b, cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemcpyAsync(C.qun + k0, f[m].qchanun, b, cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemcpyAsync(C.qvn + k0, f[m].qchanvn, b, cudaMemcpyHostToDevice, c->stream));
    }
    CK(cudaMemcpyAsync(c->chan_hp1, c->hp1_h.data(), sizeof(double) * M,
                       cudaMemcpyHostToDevice, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return EFDC_XM_OK;
}

// What the context records of an upload: which device copies are out of
// date, whether it holds the three time levels, the entry masks (OLDMASK).
// The implicit drag inputs (DRAG_*) an upload of f sends.
unsigned drag_in_of(const efdc_xm_fields *f) {
  unsigned b = 0;
  if (f[0].ubot && f[0].vbot && f[0].vu && f[0].uv && f[0].stbx && f[0].stby && f[0].uhe &&
      f[0].vhe)
    b |= DRAG_BED;
  if (f[0].fxvege && f[0].fyvege) b |= DRAG_VEG;
  return b;
}

void upload_done(efdc_xm_ctx *c, const efdc_xm_fields *f, bool skip_wetdry, bool skip_sbxy,
                 bool levels) {
  c->drag_in |= drag_in_of(f);
  c->wd_stale = skip_wetdry;
  c->sbxy_stale = skip_sbxy;
  c->tl3_ready = levels;
  if (!skip_wetdry)
    for (int m = 0; m < c->M; ++m)
      if (f[m].lmaskdry)
        c->mem[m].oldmask_h.assign(f[m].lmaskdry, f[m].lmaskdry + c->mem[m].lc);
}

int upload_batch(efdc_xm_ctx *c, const efdc_xm_fields *f, bool skip_wetdry, bool skip_sbxy,
                 bool levels) {
  if (!c || !f) {
    set_error("efdc_xm_upload: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  std::vector<Xfer> xs;
  uint32_t sent = 0;
  int rc = plan_upload(c, f, skip_wetdry, skip_sbxy, levels, xs, &sent);
  if (!rc) rc = upload_arrays(c, xs);
  if (!rc && !levels) rc = copy_levels(c, f, 0, size_t(c->nslot), c->stream);
  if (!rc) rc = upload_small(c, f);
  if (rc) {
    c->synced = 0;  // the device copies are not known to match anything
    return rc;
  }
  c->synced |= sent;
  upload_done(c, f, skip_wetdry, skip_sbxy, levels);
  return EFDC_XM_OK;
}
}  // namespace

namespace {
int download_batch(efdc_xm_ctx *c, efdc_xm_fields *f, bool skip_unchanged, int levels);
}

int32_t efdc_xm_download_batch(efdc_xm_ctx *c, efdc_xm_fields *f) {
  return download_batch(c, f, false, c && c->tl3_ready ? 3 : 0);
}

namespace {
// skip_unchanged: leave out the fields that a step with ISDRY = 0 in every
// member does not write (the face switches SUB, SVB, SBX, SBY, LMASKDRY,
// ISCDRY, NATDRY, QDWASTE, VDWASTE): within efdc_xm_step_batch their device
// values are the host values uploaded by the same call.  levels: the three
// time levels to return (0 none; 2 FPGXE, FPGYE, which a CALPUV9C(2) step
// changes; 3 all of them, after CALPUV9C(3)).
// The wet/dry lists of a download: the mask at exit and at entry (OLDMASK)
// of every member, gathered into these host copies.
struct Lists {
  bool on = false;
  std::vector<std::vector<int32_t>> mask, oldm;
};

// The arrays of a download.
// The arrays of a download; *got: the bits (enum efdc_xm_same) of those that
// come back, whose device copies then match the caller's arrays.
int plan_download(efdc_xm_ctx *c, efdc_xm_fields *f, bool skip_unchanged, int levels,
                  std::vector<Xfer> &xs, Lists &ls, uint32_t *got = nullptr) {
  xm::DevState &X = c->X;
  const xm::DevSystem &Y = c->Y;
  const int M = c->M;
  int rc = 0;
  uint32_t back = 0;
#define XM_DN(name, dev, kind)                                   \
  {                                                              \
    std::vector<const void *> v(M);                              \
    for (int m = 0; m < M; ++m) v[m] = f[m].name;                \
    if ((rc = collect(c, xs, v, dev, kind, #name))) return rc;   \
  }
#define XM_DNB(name, dev, kind, bit)                             \
  {                                                              \
    const size_t n0 = xs.size();                                 \
    XM_DN(name, dev, kind)                                       \
    if (xs.size() > n0) back |= (bit);                           \
  }
  XM_DNB(p, X.p, 0, EFDC_XM_SAME_P) XM_DNB(hp, X.hp, 0, EFDC_XM_SAME_HP) XM_DN(h1p, X.h1p, 0)
  XM_DNB(hu, X.hu, 0, EFDC_XM_SAME_HU) XM_DNB(hv, X.hv, 0, EFDC_XM_SAME_HV)
  XM_DNB(uhdye, X.uhdye, 0, EFDC_XM_SAME_UHDYE) XM_DNB(vhdxe, X.vhdxe, 0, EFDC_XM_SAME_VHDXE)
  XM_DNB(lopenbcdry, X.lopenbcdry, 1, EFDC_XM_SAME_LOPENBCDRY)
  XM_DN(uhe, X.uhe, 0) XM_DN(vhe, X.vhe, 0) XM_DN(hpi, X.hpi, 0) XM_DN(hui, X.hui, 0)
  XM_DN(hvi, X.hvi, 0)
  if (!skip_unchanged) {
    XM_DNB(sub, X.sub, 0, EFDC_XM_SAME_SUB) XM_DNB(svb, X.svb, 0, EFDC_XM_SAME_SVB)
    if (!c->sbxy_stale) {  // else the host holds them (see sbxy_stale)
      XM_DNB(sbx, X.sbx, 0, EFDC_XM_SAME_SBX) XM_DNB(sby, X.sby, 0, EFDC_XM_SAME_SBY)
    }
    if (!c->wd_stale) {
      XM_DNB(lmaskdry, X.lmaskdry, 1, EFDC_XM_SAME_LMASKDRY)
      XM_DNB(iscdry, X.iscdry, 2, EFDC_XM_SAME_ISCDRY)
      XM_DNB(natdry, X.natdry, 2, EFDC_XM_SAME_NATDRY)
      XM_DNB(qdwaste, X.qdwaste, 0, EFDC_XM_SAME_QDWASTE)
      XM_DNB(vdwaste, X.vdwaste, 0, EFDC_XM_SAME_VDWASTE)
    }
  }
  if (got) *got = back;
#undef XM_DNB
  XM_DN(ccc, Y.ccc, 0) XM_DN(ccs, Y.ccs, 0) XM_DN(ccw, Y.ccw, 0) XM_DN(cce, Y.cce, 0)
  XM_DN(ccn, Y.ccn, 0) XM_DN(fptmp, Y.fptmp, 0)
  if (levels && c->tl3_alloc) {
    XM_DN(fpgxe, X.fpgxe, 0) XM_DN(fpgye, X.fpgye, 0)
    if (levels == 3) {
      XM_DN(p1, X.p1, 0) XM_DN(h2p, X.h2p, 0) XM_DN(uhdy1e, X.uhdy1e, 0)
      XM_DN(vhdx1e, X.vhdx1e, 0) XM_DN(uhdy2e, X.uhdy2e, 0) XM_DN(vhdx2e, X.vhdx2e, 0)
      XM_DN(h1u, X.h1u, 0) XM_DN(h1v, X.h1v, 0)
    }
  }
#undef XM_DN
  // the wet/dry lists need the mask at exit and at entry (OLDMASK)
  ls.mask.assign(M, {});
  ls.oldm.assign(M, {});
  ls.on = false;
  for (int m = 0; m < M; ++m) ls.on |= (f[m].lwet || f[m].ldry);
  if (ls.on) {
    std::vector<const void *> pm(M), po(M);
    for (int m = 0; m < M; ++m) {
      ls.mask[m].assign(c->mem[m].lc, 1);
      ls.oldm[m].assign(c->mem[m].lc, 1);
      pm[m] = ls.mask[m].data();
      po[m] = ls.oldm[m].data();
    }
    xs.push_back(Xfer{pm, X.lmaskdry, 1});
    xs.push_back(Xfer{po, X.oldmask, 2});
  }
  return EFDC_XM_OK;
}

// After the arrays of a download: the channels' flows, and the wet/dry lists
// from the gathered masks (calpuv2c.f90:1061-1080, L order).
int download_finish(efdc_xm_ctx *c, efdc_xm_fields *f, const Lists &ls) {
  const int M = c->M;
  if (c->S.ch.n > 0) {
    const xm::DevChan &C = c->S.ch;
    for (int m = 0; m < M; ++m) {
      const int k0 = c->chan_start[m], n = c->chan_start[m + 1] - k0;
      if (n == 0) continue;
      const size_t b = sizeof(double) * size_t(n);
      if (f[m].qchanu) CK(cudaMemcpyAsync(f[m].qchanu, C.qu + k0, b, cudaMemcpyDeviceToHost, c->stream));
      if (f[m].qchanv) CK(cudaMemcpyAsync(f[m].qchanv, C.qv + k0, b, cudaMemcpyDeviceToHost, c->stream));
      if (f[m].qchanun)
        CK(cudaMemcpyAsync(f[m].qchanun, C.qun + k0, b, cudaMemcpyDeviceToHost, c->stream));
      if (f[m].qchanvn)
        CK(cudaMemcpyAsync(f[m].qchanvn, C.qvn + k0, b, cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
  }
  if (ls.on) {
    for (int m = 0; m < M; ++m) {
      const Member &mb = c->mem[m];
      int nw = 0, nd = 0;
      for (int L = 2; L <= mb.la; ++L) {
        if (mb.last_isdry == 0 || ls.mask[m][L - 1]) {
          if (f[m].lwet) f[m].lwet[nw] = L;
          ++nw;
        } else if (ls.oldm[m][L - 1] || mb.last_n < mb.last_ntstbc + 1) {
          if (f[m].ldry) f[m].ldry[nd] = L;
          ++nd;
        }
      }
    }
  }
  return EFDC_XM_OK;
}

bool wants_system(const efdc_xm_fields *f) {
  return f[0].ccc || f[0].ccs || f[0].ccw || f[0].cce || f[0].ccn || f[0].fptmp;
}

int download_batch(efdc_xm_ctx *c, efdc_xm_fields *f, bool skip_unchanged, int levels) {
  if (!c || !f) {
    set_error("efdc_xm_download: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  std::vector<Xfer> xs;
  Lists ls;
  uint32_t got = 0;
  int rc = plan_download(c, f, skip_unchanged, levels, xs, ls, &got);
  if (rc) return rc;
  if (c->last_mixed && wants_system(f)) {
    // a MIXED step solves from the unscaled assembly: the scaled system
    // (calpuv2c.f90:371-399) is formed when it is asked for
    if ((rc = scaled_system(c))) return rc;
  }
  if (f[0].hpi || f[0].hui || f[0].hvi) {  // 1/HP, 1/HU, 1/HV are formed on request
    xm::launch_reciprocals(c->L(), c->S, c->X, 1, c->ntile);
    CK(cudaGetLastError());
  }
  if ((rc = download_arrays(c, xs))) return rc;
  c->synced |= got;
  return download_finish(c, f, ls);
}
}  // namespace

}  // extern "C"

namespace {
// ---------------------------------------------------------------------------
// Device-driven step: one CALPUV2C (or CALPUV9C) call of every active member
// as one CUDA graph.  The three data-dependent loops of the step -- the CG
// iterations, the MIXED refinement passes with their inner iterations, and
// the wet/dry re-solves -- are conditional WHILE nodes whose conditions the
// loop-control kernels (xm_loop.cu) set on the device, so the host launches
// the graph and waits once, for the stats.  Every loop has a body cap on the
// device (ITERM-based for the solves, the members' NCORDRY cap for the
// sweeps, MAX_OUTER for the passes).  The graph holds the kernels' arguments,
// so it is cached by the bytes of every view it was built from (the two-level
// buffer swap alternates between two such graphs).

// What a step's graph depends on besides the context's device views.
struct StepPlan {
  int mixed, istl, all, any_isdry, any_legacy, any99, any_waste, iters;
  int max_iterm, max_sweeps, grid, grid_cg, grid_cg32, grid_up32;
  int mx_jac, mx_poly, may_asym, chan, baro, obc_serial, any_may_asym, nmember;
  int variant, ctas_mv, ctas_up, any_drag, small;
  double fac, inner_margin;
  const void *psol;
};

template <class T>
void put_bytes(std::vector<char> &k, const T &v) {
  const char *p = reinterpret_cast<const char *>(&v);
  k.insert(k.end(), p, p + sizeof(T));
}

// The key of a step graph: the plan and every view its kernels take (DevState,
// DevSystem and DevObc hold pointers and ints only, no padding; DevStatic
// changes only through the set-up calls, which drop the graphs).
std::vector<char> step_key(const efdc_xm_ctx *c, const StepPlan &pl) {
  std::vector<char> k;
  k.reserve(2048);
  put_bytes(k, pl);
  put_bytes(k, c->X);
  put_bytes(k, c->Y);
  put_bytes(k, c->B);
  for (const void *p : {static_cast<const void *>(c->mxview.fp), static_cast<const void *>(c->mxview.cc),
                        static_cast<const void *>(c->mxview.cs), static_cast<const void *>(c->mxview.cw),
                        static_cast<const void *>(c->mxview.ce), static_cast<const void *>(c->mxview.cn)})
    put_bytes(k, p);
  put_bytes(k, c->mxview.unscaled);
  return k;
}

// A conditional handle in the graph now being captured on `st`.
cudaError_t cond_handle(cudaStream_t st, cudaGraphConditionalHandle *h) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr);
  if (e != cudaSuccess) return e;
  if (cs != cudaStreamCaptureStatusActive || !g) return cudaErrorStreamCaptureInvalidated;
  return cudaGraphConditionalHandleCreate(h, g, 0, 0);
}

// Appends a WHILE node with handle h at the current end of the capture on
// `st` (later work on `st` follows it) and starts capturing its body on `bs`.
cudaError_t begin_while(cudaStream_t st, cudaGraphConditionalHandle h, cudaStream_t bs) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd);
  if (e != cudaSuccess) return e;
  cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};  // the rest zero
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  if ((e = cudaGraphAddNode(&node, g, deps, nd, &p)) != cudaSuccess) return e;
  if ((e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies)) !=
      cudaSuccess)
    return e;
  return cudaStreamBeginCaptureToGraph(bs, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                       cudaStreamCaptureModeThreadLocal);
}

cudaError_t end_body(cudaStream_t bs) {
  cudaGraph_t g = nullptr;
  return cudaStreamEndCapture(bs, &g);
}

// Records the kernels launched since `*mark` into `*n` and moves the mark.
void take_count(long long *mark, long long *n) {
  const long long now = g_launches.load();
  *n += now - *mark;
  *mark = now;
}

#define CKG(expr)                        \
  do {                                   \
    const cudaError_t e__ = (expr);      \
    if (e__ != cudaSuccess) return e__; \
  } while (0)

// The solve of one sweep, captured on level d (stream c->cap_stream[d]).
cudaError_t capture_solve(efdc_xm_ctx *c, const StepPlan &pl, int d, StepGraph &sg,
                          long long *mark, long long *mine) {
  cudaStream_t st = c->cap_stream[d];
  xm::Launch l = c->L();
  l.stream = st;
  const int M = c->M, K = pl.iters;
  double *P = c->X.p;
  if (!pl.mixed && pl.small) {  // one CTA per member, its loop inside (k_cg_small)
    xm::launch_solve_reset(l, c->ctl, c->glob, c->act, M);
    xm::launch_cg_small(l, c->S, c->Y, P, c->ctl, c->glob, c->part, c->small_slots,
                        c->small_units, M);
    take_count(mark, mine);
    return cudaGetLastError();
  }
  if (!pl.mixed) {
    xm::launch_solve_reset(l, c->ctl, c->glob, c->act, M);
    xm::launch_cg_init(l, c->S, c->Y, P, c->ctl, c->glob, c->part);
    cudaGraphConditionalHandle h;
    CKG(cond_handle(st, &h));
    xm::launch_loop_enter(st, c->glob, xm::LOOP_CG, h, 1, M);
    take_count(mark, mine);
    CKG(begin_while(st, h, c->cap_stream[d + 1]));
    xm::Launch lb = l;
    lb.stream = c->cap_stream[d + 1];
    for (int k = 0; k < K; ++k) xm::launch_cg_iter(lb, c->S, c->Y, P, c->ctl, c->glob, c->part);
    xm::launch_loop_next(lb.stream, c->glob, xm::LOOP_CG, h, (pl.max_iterm + K - 1) / K + 1, 0,
                         M);
    take_count(mark, &sg.n_body[xm::LOOP_CG]);
    CKG(end_body(lb.stream));
    xm::launch_cg_finish(l, c->S, c->Y, P, c->ctl);  // the last iteration's P += alpha*p
    take_count(mark, mine);
    return cudaGetLastError();
  }
  xm::launch_solve_reset(l, c->ctl, c->glob, c->act, M);
  xm::launch_chan_p0(l, c->S, c->mxview, P, c->act);
  cudaGraphConditionalHandle ho, hi;
  CKG(cond_handle(st, &ho));
  xm::launch_loop_enter(st, c->glob, xm::LOOP_OUTER, ho, 0, M);
  take_count(mark, mine);
  CKG(begin_while(st, ho, c->cap_stream[d + 1]));
  xm::Launch lo = l;
  lo.stream = c->cap_stream[d + 1];
  xm::launch_outer_reset(lo, c->glob);
  xm::launch_mx_resid(lo, c->S, c->mxview, c->Y, P, c->ctl, c->glob, c->part, pl.fac,
                      inner_rel_tol(c), 0);
  CKG(cond_handle(lo.stream, &hi));
  xm::launch_loop_enter(lo.stream, c->glob, xm::LOOP_INNER, hi, 1, M);
  take_count(mark, &sg.n_body[xm::LOOP_OUTER]);
  CKG(begin_while(lo.stream, hi, c->cap_stream[d + 2]));
  xm::Launch li = l;
  li.stream = c->cap_stream[d + 2];
  for (int k = 0; k < K; ++k) xm::launch_mx_iter(li, c->S, c->Y, c->ctl, c->glob, c->part);
  // the inner stop caps each member at 2*ITERM+50 inner iterations in all
  xm::launch_loop_next(li.stream, c->glob, xm::LOOP_INNER, hi,
                       (2 * pl.max_iterm + 50 + K - 1) / K + 2, 1, M);
  take_count(mark, &sg.n_body[xm::LOOP_INNER]);
  CKG(end_body(li.stream));
  xm::launch_inner_done(lo.stream, c->ctl, c->act, M);
  xm::launch_mx_apply(lo, c->S, c->mxview, c->Y, P, c->ctl);
  xm::launch_loop_next(lo.stream, c->glob, xm::LOOP_OUTER, ho, MAX_OUTER, 0, M);
  take_count(mark, &sg.n_body[xm::LOOP_OUTER]);
  return end_body(lo.stream);
}

// Captures the whole step into sg (the host has set the views, the swaps,
// the scalars and the members' activity; see step_range).
// x_pre: the state views before the time-level rotation of CALPUV9C(3), on
// which its first kernels run (as in step_range's host-driven order).
cudaError_t capture_step(efdc_xm_ctx *c, const StepPlan &pl, const xm::DevState &x_pre,
                         StepGraph &sg) {
  for (cudaStream_t &s : c->cap_stream)
    if (!s) CKG(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  cudaStream_t s0 = c->cap_stream[0], s1 = c->cap_stream[1];
  const int M = c->M;
  xm::Launch l = c->L();
  l.stream = s0;
  long long mark = g_launches.load();
  const long long start = mark;
  CKG(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  [&] {
    xm::launch_step_enter(s0, c->ctl, c->act, c->glob, M);
    if (pl.istl == 0) {
      xm::launch_chan_entry(l, c->S, c->X, c->act);
      xm::launch_begin(l, c->S, c->X, c->act, !pl.all);
      if (pl.any_drag) xm::launch_implicit_drag(l, c->S, c->X, c->act);
    } else {
      xm::launch_chan_entry(l, c->S, x_pre, c->act);
      xm::launch_begin3(l, c->S, x_pre, c->act);
      if (pl.any_drag) xm::launch_implicit_drag(l, c->S, x_pre, c->act);
      if (pl.istl == 3) xm::launch_advance3(l, c->S, c->X);
    }
    if (pl.any_isdry) xm::launch_obc_reset(l, c->S, c->B, c->X, c->act);
    cudaGraphConditionalHandle hs;
    if ((err = cond_handle(s0, &hs)) != cudaSuccess) return;
    xm::launch_loop_enter(s0, c->glob, xm::LOOP_SWEEP, hs, 0, M);
    take_count(&mark, &sg.n_top);
    if ((err = begin_while(s0, hs, s1)) != cudaSuccess) return;
    // the sweep body (1000 CONTINUE of calpuv2c.f90)
    xm::Launch lw = l;
    lw.stream = s1;
    xm::launch_sweep_reset(lw, c->ctl, c->act, M);
    xm::launch_assemble(lw, c->S, c->X, c->ctl, c->act);
    xm::launch_obc(lw, c->S, c->X, c->B, c->ctl, c->act, c->obc_serial, c->any_may_asym ? 1 : 0);
    xm::launch_chan_sub(lw, c->S, c->X, c->ctl, c->act, -1);
    xm::launch_scale(lw, c->S, c->X, c->Y, c->ctl, c->act, pl.mixed, c->any_may_asym ? 1 : 0);
    if ((err = capture_solve(c, pl, 1, sg, &mark, &sg.n_body[xm::LOOP_SWEEP])) != cudaSuccess)
      return;
    if (c->psol) {  // calibration: the adjoint needs P' before P is refreshed from HP
      if ((err = cudaMemcpyAsync(c->psol, c->X.p, size_t(c->nslot) * sizeof(double),
                                 cudaMemcpyDeviceToDevice, s1)) != cudaSuccess)
        return;
    }
    xm::launch_after_solve(s1, c->ctl, c->act, M, pl.mixed);
    xm::launch_chan_flow(lw, c->S, c->X, c->act);
    xm::launch_backsub(lw, c->S, c->X, c->act);
    xm::launch_obc_hp(lw, c->S, c->X, c->B, c->act);
    xm::launch_chan_exch(lw, c->S, c->X, c->act);
    if (pl.any_isdry) xm::launch_wetdry(lw, c->S, c->X, c->ctl, c->act, pl.any_legacy, pl.any99);
    xm::launch_sweep_next(s1, c->S, c->ctl, c->act, c->glob, hs, pl.max_sweeps + 1, M);
    take_count(&mark, &sg.n_body[xm::LOOP_SWEEP]);
    if ((err = end_body(s1)) != cudaSuccess) return;
    // finalisation of the members whose sweeps ended normally
    xm::launch_fin_prepare(s0, c->ctl, c->act, M);
    xm::launch_final(l, c->S, c->X, c->ctl, c->act, pl.any_waste);
    take_count(&mark, &sg.n_top);
  }();
  cudaGraph_t g = nullptr;
  const cudaError_t e_end = cudaStreamEndCapture(s0, &g);
  // captured, not launched: the step's launches are counted when it runs
  g_launches.fetch_sub(g_launches.load() - start);
  if (err == cudaSuccess) err = e_end;
  if (err == cudaSuccess && !g) err = cudaErrorStreamCaptureInvalidated;
  if (err == cudaSuccess) err = cudaGraphInstantiate(&sg.exec, g, 0);
  if (g) cudaGraphDestroy(g);
  if (err != cudaSuccess) {
    // a capture left open on a body stream would keep that stream capturing
    for (cudaStream_t s : c->cap_stream) {
      cudaStreamCaptureStatus cs;
      if (s && cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t t = nullptr;
        cudaStreamEndCapture(s, &t);
        if (t) cudaGraphDestroy(t);
      }
    }
    cudaGetLastError();
    sg.exec = nullptr;
  }
  return err;
}
#undef CKG

constexpr size_t STEP_GRAPH_CACHE = 8;

// The cached graph for this step, built on first use; null if graphs with
// conditional nodes cannot be built here (the host-driven step then runs).
StepGraph *step_graph(efdc_xm_ctx *c, const StepPlan &pl, const xm::DevState &x_pre) {
  std::vector<char> key = step_key(c, pl);
  if (pl.istl != 0) put_bytes(key, x_pre);
  for (size_t i = 0; i < c->step_graphs.size(); ++i)
    if (c->step_graphs[i].key == key) {
      if (i + 1 != c->step_graphs.size())  // most recent last
        std::rotate(c->step_graphs.begin() + i, c->step_graphs.begin() + i + 1,
                    c->step_graphs.end());
      return &c->step_graphs.back();
    }
  for (const auto &f : c->step_graph_failed)
    if (f == key) return nullptr;
  StepGraph sg;
  if (capture_step(c, pl, x_pre, sg) != cudaSuccess || !sg.exec) {
    c->step_graph_failed.push_back(std::move(key));
    return nullptr;
  }
  sg.key = std::move(key);
  if (c->step_graphs.size() >= STEP_GRAPH_CACHE) {
    cudaGraphExecDestroy(c->step_graphs.front().exec);
    c->step_graphs.erase(c->step_graphs.begin());
  }
  c->step_graphs.push_back(std::move(sg));
  return &c->step_graphs.back();
}

void drop_step_graphs(efdc_xm_ctx *c) {
  for (StepGraph &g : c->step_graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  c->step_graphs.clear();
  c->step_graph_failed.clear();
}

// A bounded wait in a kernel ran out (Glob::err): every member of the step
// fails with EFDC_XM_DEVICE_TIMEOUT; the flag is cleared for the next call.
int device_timeout(efdc_xm_ctx *c, efdc_xm_stats *stats, int m0, int m1) {
  set_error("a bounded device-side wait ran out (bulk copies into shared memory did not "
            "complete); the step's results are not valid");
  for (int m = m0; m < m1; ++m) stats[m].status = EFDC_XM_DEVICE_TIMEOUT;
  CK(cudaMemsetAsync(&c->glob->err, 0, sizeof(int), c->stream));
  return EFDC_XM_DEVICE_TIMEOUT;
}

// Runs the step's graph and reads the members' control blocks (one host
// wait), then fills the stats of the members [m0, m1) as step_range's host
// loop does.  Returns -1 (nothing launched) if the graph could not be built.
int run_step_graph(efdc_xm_ctx *c, const StepPlan &pl, const xm::DevState &x_pre,
                   const efdc_xm_params *prm, efdc_xm_stats *stats, int m0, int m1) {
  StepGraph *sg = step_graph(c, pl, x_pre);
  if (!sg) return -1;
  CK(cudaGraphLaunch(sg->exec, c->stream));
  if (c->in_chunks && c->ctl_hd && c->glob_hd) {
    xm::launch_words(c->stream, c->ctl_hd, c->ctl, sizeof(Ctl) * c->M);
    xm::launch_words(c->stream, c->glob_hd, c->glob, sizeof(Glob));
  } else {
    CK(cudaMemcpyAsync(c->ctl_h, c->ctl, sizeof(Ctl) * c->M, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(c->glob_h, c->glob, sizeof(Glob), cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  g_waits.fetch_add(1, std::memory_order_relaxed);
  long long n = sg->n_top;
  for (int i = 0; i < xm::NLOOP; ++i) n += sg->n_body[i] * c->glob_h->tot[i];
  xm::count_launches(int(std::min<long long>(n, INT32_MAX)));
  if (c->glob_h->err) return device_timeout(c, stats, m0, m1);
  for (int m = m0; m < m1; ++m) {
    const Ctl &k = c->ctl_h[m];
    efdc_xm_stats &s = stats[m];
    Member &mb = c->mem[m];
    s.iters_last = k.iters_last;
    s.iters_total += k.iters_total;
    s.solves += k.solves;
    s.rsq_last = k.rsq_last;
    s.outer_refinements += k.outer_total;
    s.ccmnm_last = k.ccmnm_last;
    s.n_negdep = k.nneg;
    s.n_wasted = k.nwasted;
    if (k.iters_last > 0) mb.last_iters = k.iters_last;
    if (pl.mixed && k.last_inner > 0) mb.last_inner = k.last_inner;
    if (pl.mixed && k.inner_first > 0) {
      const bool poly = c->mpoly_h[m] && !(k.asym & 1);
      mb.jac_est = float(k.inner_first) * (poly ? 1.9f : 1.0f);
    }
    int st = k.mstatus;
    if (st == EFDC_XM_UNSUPPORTED) {
      set_error("member %d: the scaled operator is unsymmetric although the model has no "
                "radiation boundary (check SUBO/SVBO next to the open-boundary cells)", m);
    } else if (st == EFDC_XM_CG_MAXITER || (st == EFDC_XM_NONFINITE && k.status == st)) {
      set_error("member %d: CONGRAD: %s after %d iterations (RSQ=%g, RSQM=%g)", m,
                st == EFDC_XM_CG_MAXITER ? "maximum iterations exceeded" : "non-finite residual",
                k.iter, s.rsq_last, prm[m].rsqm);
    } else if (st == EFDC_XM_WETDRY_MAXSWEEP) {
      set_error("member %d: wet/dry: NCORDRY reached %d", m, c->sc_h[m].max_sweeps);
    }
    if (st == EFDC_XM_OK && k.nnonfinite > 0) {
      st = EFDC_XM_NONFINITE;
      set_error("member %d: non-finite P in %d cells", m, k.nnonfinite);
    }
    if (st == EFDC_XM_OK && k.nneg > 0) st = EFDC_XM_NEG_DEPTH;
    s.status = st;
  }
  return overall_status(stats + m0, m1 - m0);
}

}  // namespace
extern "C" {
namespace {
void drop_graphs(efdc_xm_ctx *c);  // (below, where it is defined with C linkage)
}  // namespace
}  // extern "C"
namespace {

// ---------------------------------------------------------------------------
// Schedule autotuner (efdc_xm_autotune).  The reference's only schedule rule
// is its thread count, NOPTIMAL = MIN(NTHREADS, 8, MAX(LA/100, 1))
// (calpuv2c.f90:61-62); here the knobs are the MIXED inner iteration's kernel
// variant and CTA caps, the CG iterations per loop body, the Jacobi /
// polynomial threshold and the inner target margin and tolerance.  The tuner times the
// context's own solve -- the solve part of a device-driven step, captured as
// a graph of the same kernels -- on the system the last step assembled, from
// the P it left (restored before every run), and walks the knobs one at a
// time (coordinate descent, each knob's candidates in a fixed order, the
// first of equal times kept), so the same measurements give the same choice.

constexpr int TUNE_REPS = 5;          // timed solves per candidate (the median counts)
constexpr double TUNE_GAIN = 0.98;    // a candidate must be 2 % faster to replace the incumbent
constexpr double TUNE_MIN_MS = 20.0;  // timed solve time per candidate sought (see tune_time)

void schedule_of(const efdc_xm_ctx *c, efdc_xm_schedule *s) {
  s->kernel_variant = c->kvariant;
  s->ctas_matvec = c->ctas_mv;
  s->ctas_update = c->ctas_up;
  s->graph_iters = c->graph_iters;
  s->poly_threshold = int32_t(c->poly_threshold);
  s->inner_margin = c->inner_margin_log10;
  s->inner_tol = c->inner_tol_x10;
}

void apply_schedule(efdc_xm_ctx *c, const efdc_xm_schedule &s) {
  if (s.kernel_variant != c->kvariant || s.ctas_matvec != c->ctas_mv ||
      s.ctas_update != c->ctas_up || s.inner_margin != c->inner_margin_log10 ||
      s.graph_iters != c->graph_iters || s.inner_tol != c->inner_tol_x10)
    drop_graphs(c);
  c->kvariant = s.kernel_variant;
  c->ctas_mv = s.ctas_matvec;
  c->ctas_up = s.ctas_update;
  c->graph_iters = s.graph_iters;
  c->poly_threshold = float(s.poly_threshold);
  c->inner_margin_log10 = s.inner_margin;
  c->inner_tol_x10 = s.inner_tol;
}

bool schedule_valid(const efdc_xm_schedule &s) {
  return s.kernel_variant >= 0 && s.kernel_variant <= 3 && s.ctas_matvec >= 0 &&
         s.ctas_matvec <= 32 && s.ctas_update >= 0 && s.ctas_update <= 32 &&
         s.graph_iters >= 1 && s.graph_iters <= 32 && s.poly_threshold >= 0 &&
         s.poly_threshold <= 100000 && s.inner_margin >= 0 && s.inner_margin <= 6 &&
         s.inner_tol >= 40 && s.inner_tol <= 75;
}

// The workload key of a table line: the precision, the buckets (floor log2)
// of the member count and of the water cells, and the operator's form.
std::string tune_key(const efdc_xm_ctx *c, int precision) {
  long long cells = 0;
  for (const Member &mb : c->mem) cells += mb.la - 1;
  auto lg = [](long long v) {
    int b = 0;
    while (v > 1) {
      v >>= 1;
      ++b;
    }
    return b;
  };
  char buf[160];
  snprintf(buf, sizeof(buf), "prec=%s members=2^%d cells=2^%d asym=%d chan=%d",
           precision == EFDC_XM_PREC_MIXED ? "mixed" : "fp64", lg(c->M), lg(cells),
           c->any_may_asym ? 1 : 0, c->S.ch.n > 0 ? 1 : 0);
  return buf;
}

// "key | variant=.. ctas_mv=.. ctas_up=.. iters=.. poly=.. margin=.. tol=.. | ms=.."
std::string table_line(const std::string &key, const efdc_xm_schedule &s, double ms) {
  char buf[400];
  snprintf(buf, sizeof(buf),
           "%s | variant=%d ctas_mv=%d ctas_up=%d iters=%d poly=%d margin=%d tol=%d | ms=%.4f",
           key.c_str(), s.kernel_variant, s.ctas_matvec, s.ctas_update, s.graph_iters,
           s.poly_threshold, s.inner_margin, s.inner_tol, ms);
  return buf;
}

// The schedule of the last line of the table whose key is `key`.
bool table_lookup(const char *path, const std::string &key, efdc_xm_schedule *out) {
  FILE *f = path ? fopen(path, "r") : nullptr;
  if (!f) return false;
  char line[1024];
  bool found = false;
  while (fgets(line, sizeof(line), f)) {
    std::string l(line);
    const size_t bar = l.find(" | ");
    if (bar == std::string::npos || l.compare(0, bar, key) != 0 || bar != key.size()) continue;
    efdc_xm_schedule s{};
    s.inner_tol = 60;  // lines written before the tolerance was a knob
    const int n = sscanf(l.c_str() + bar + 3,
                         "variant=%d ctas_mv=%d ctas_up=%d iters=%d poly=%d margin=%d tol=%d",
                         &s.kernel_variant, &s.ctas_matvec, &s.ctas_update, &s.graph_iters,
                         &s.poly_threshold, &s.inner_margin, &s.inner_tol);
    if (n >= 6 && schedule_valid(s)) {
      *out = s;
      found = true;
    }
  }
  fclose(f);
  return found;
}

// The solve of every member as a graph (the solve part of a step's graph).
cudaError_t capture_solve_graph(efdc_xm_ctx *c, const StepPlan &pl, cudaGraphExec_t *exec) {
  for (cudaStream_t &s : c->cap_stream)
    if (!s) {
      const cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
      if (e != cudaSuccess) return e;
    }
  StepGraph sg;
  long long mark = g_launches.load();
  const long long start = mark;
  long long mine = 0;
  cudaError_t err = cudaStreamBeginCapture(c->cap_stream[0], cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) return err;
  err = capture_solve(c, pl, 0, sg, &mark, &mine);
  cudaGraph_t g = nullptr;
  const cudaError_t e_end = cudaStreamEndCapture(c->cap_stream[0], &g);
  g_launches.fetch_sub(g_launches.load() - start);
  if (err == cudaSuccess) err = e_end;
  if (err == cudaSuccess && !g) err = cudaErrorStreamCaptureInvalidated;
  if (err == cudaSuccess) err = cudaGraphInstantiate(exec, g, 0);
  if (g) cudaGraphDestroy(g);
  if (err != cudaSuccess) {
    for (cudaStream_t s : c->cap_stream) {
      cudaStreamCaptureStatus cs;
      if (s && cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t t = nullptr;
        cudaStreamEndCapture(s, &t);
        if (t) cudaGraphDestroy(t);
      }
    }
    cudaGetLastError();
    *exec = nullptr;
  }
  return err;
}

// Median device time of `reps` solves of every member under the context's
// current schedule, each from the saved P (*ms < 0: the schedule failed).
int tune_time(efdc_xm_ctx *c, bool mixed, double fac, int reps, double *ms) {
  *ms = -1.0;
  for (int m = 0; m < c->M; ++m) c->act_h[m] = 1;
  int rc = write_act(c);
  if (rc) return rc;
  if (mixed && (rc = choose_inner(c))) return rc;
  const xm::Launch lk = c->L();
  StepPlan pl{};
  pl.mixed = mixed;
  pl.small = !mixed && small_solve(c);
  pl.iters = c->graph_iters;
  pl.max_iterm = 1;
  for (int m = 0; m < c->M; ++m) pl.max_iterm = std::max(pl.max_iterm, c->sc_h[m].iterm);
  pl.fac = fac;
  pl.inner_margin = lk.inner_margin;
  pl.nmember = c->M;
  cudaGraphExec_t ex = nullptr;
  if (capture_solve_graph(c, pl, &ex) != cudaSuccess || !ex) return EFDC_XM_OK;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const size_t pb = size_t(c->nslot) * sizeof(double);
  std::vector<double> t;
  int n = reps;
  for (int r = 0; r <= n; ++r) {  // run 0 warms up
    CK(cudaMemcpyAsync(c->X.p, c->ptmp, pb, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaEventRecord(e0, c->stream));
    CK(cudaGraphLaunch(ex, c->stream));
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, e0, e1));
    if (r > 0) t.push_back(f);
    // short solves take more runs (about TUNE_MIN_MS of them, up to 4x reps):
    // their run-to-run spread is a larger share of their time
    if (r == 0 && f > 0.f) n = std::min(4 * reps, std::max(reps, int(TUNE_MIN_MS / f) + 1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaGraphExecDestroy(ex);
  if ((rc = read_glob(c))) return rc;
  if (c->glob_h->err) {  // a bounded wait ran out: this schedule is not usable here
    CK(cudaMemsetAsync(&c->glob->err, 0, sizeof(int), c->stream));
    return EFDC_XM_OK;
  }
  std::sort(t.begin(), t.end());
  *ms = t[t.size() / 2];
  return EFDC_XM_OK;
}

// The argument checks of a device-resident step of every member (the stats
// are filled with the status on failure).
int validate_step(efdc_xm_ctx *c, const efdc_xm_params *prm, efdc_xm_stats *stats) {
  const int M = c->M;
  for (int m = 0; m < M; ++m) {
    if (!(prm[m].delt > 0) || prm[m].iterm < 1 || prm[m].g <= 0) {
      set_error("efdc_xm_step_device: member %d: need DELT > 0, G > 0, ITERM >= 1", m);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
    if ((prm[m].precision != EFDC_XM_PREC_FP64 && prm[m].precision != EFDC_XM_PREC_MIXED) ||
        prm[m].precision != prm[0].precision) {
      set_error("efdc_xm_step_device: member %d: unknown precision %d, or members differ", m,
                prm[m].precision);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
  }
  const int istl = prm[0].tl3_istl;  // 0: CALPUV2C; 3, 2: CALPUV9C(ISTL_)
  for (int m = 0; m < M; ++m)
    if (prm[m].tl3_istl != istl || (istl != 0 && istl != 2 && istl != 3)) {
      set_error("efdc_xm_step_device: member %d: tl3_istl %d: need 0, 2 or 3, the same for "
                "every member of a batch", m, prm[m].tl3_istl);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
  if (istl != 0 && (!c->tl3_ready || c->calib)) {
    set_error(c->calib ? "efdc_xm_step_device: the calibration covers CALPUV2C only"
                       : "efdc_xm_step_device: CALPUV9C needs the three time levels on the "
                         "device: upload them (P1, H2P, H1P, UHDY1E, ..., H1V) first");
    fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
    return EFDC_XM_BAD_ARGUMENT;
  }
  for (int m = 0; m < M; ++m)
    if ((prm[m].isdry > 0 && (c->wd_stale || c->sbxy_stale)) ||
        (prm[m].bsc > 1.E-6 && c->sbxy_stale)) {
      set_error("efdc_xm_step_device: member %d has ISDRY > 0 or BSC > 0, but fields it reads "
                "(of SBX, SBY, LMASKDRY, ISCDRY, NATDRY, QDWASTE, VDWASTE) were last left on "
                "the host by a step without them: upload them first", m);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
  for (int m = 0; m < M; ++m)
    if ((prm[m].isitb >= 1 && !(c->drag_in & DRAG_BED)) ||
        (prm[m].isitb < 1 && prm[m].isveg > 0 && !(c->drag_in & DRAG_VEG))) {
      set_error("efdc_xm_step: member %d: ISITB >= 1 needs UBOT, VBOT, VU, UV, STBX, STBY, UHE "
                "and VHE (FXVEGE, FYVEGE optional), ISVEG > 0 alone FXVEGE and FYVEGE, "
                "uploaded with the fields", m);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
  for (int m = 0; m < M; ++m) {
    if (!(prm[m].bsc > 1.E-6)) continue;
    if (!c->has_layers[m]) {
      set_error("efdc_xm_step: member %d: BSC > 1E-6 needs the layers (efdc_xm_set_layers)", m);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
  }
  return EFDC_XM_OK;
}

// One device-resident step of the members [m0, m1); the others take no part
// (every kernel skips them) and keep their state and stats.
int step_range(efdc_xm_ctx *c, const efdc_xm_params *prm, efdc_xm_stats *stats, int m0, int m1) {
  const int M = c->M;
  const int istl = prm[m0].tl3_istl;  // 0: CALPUV2C; 3, 2: CALPUV9C(ISTL_)
  CK(cudaSetDevice(c->device));
  const bool mixed = prm[0].precision == EFDC_XM_PREC_MIXED;
  c->mxview = xm::SysView{c->X.fp, c->X.cc, c->X.cs, c->X.cw, c->X.ce, c->X.cn, 1};
  c->last_mixed = mixed;
  c->sys_external = false;
  c->step_baro = false;
  for (int m = m0; m < m1; ++m) c->step_baro |= prm[m].bsc > 1.E-6;
  const xm::Launch l = c->L();
  bool any_isdry = false, any_legacy = false, any99 = false, any_waste = false,
       any_drag = false;
  std::vector<int> ncordry(M, 0), status(M, EFDC_XM_OK), max_sweeps(M, 500);
  for (int m = 0; m < M; ++m) c->act_h[m] = 0;
  for (int m = m0; m < m1; ++m) {
    Member &mb = c->mem[m];
    c->sc_h[m] = make_scalars(mb, &prm[m]);
    mb.last_n = prm[m].n;
    mb.last_ntstbc = prm[m].ntstbc;
    mb.last_isdry = prm[m].isdry;
    max_sweeps[m] = prm[m].max_sweeps > 0 ? prm[m].max_sweeps : 500;
    const int isd = prm[m].isdry;
    any_isdry |= isd > 0;
    any_legacy |= (isd > 0 && isd != 99);
    any99 |= isd == 99;
    any_waste |= (isd > 0 && prm[m].ndrystp < 0);
    any_drag |= prm[m].isitb >= 1 || prm[m].isveg > 0;
    c->act_h[m] = 1;
  }
  // what the step writes no longer matches the caller's arrays
  c->synced &= ~(any_isdry ? STEP_WRITES : STEP_WRITES_DRYFREE);
  int rc = to_device(c, c->sc, c->sc_h, c->sc_hd, sizeof(xm::StepScalars) * M);
  if (rc) return rc;
  if (c->in_chunks)  // counters of this step (no copy engine: see to_device)
    xm::launch_words(c->stream, c->ctl, nullptr, sizeof(Ctl) * M);
  else
    CK(cudaMemsetAsync(c->ctl, 0, sizeof(Ctl) * M, c->stream));
  rc = write_act(c);
  if (rc) return rc;
  // the two-level advance UHDY1E=UHDYE, VHDX1E=VHDXE, H1P=HP
  // (calpuv2c.f90:256-264): a buffer swap when every member steps (then the
  // others are rewritten for every water cell before they are read), per-cell
  // copies in k_begin when a subset does, and always inside a chunked
  // efdc_xm_step_batch, whose download was planned on the buffers as they are
  // before the steps
  const bool all = istl == 0 && m0 == 0 && m1 == M && !c->in_chunks;
  const xm::DevState x_pre = c->X;  // CALPUV9C's first kernels run before the rotation
  if (istl == 0) {
    if (all) {
      std::swap(c->X.uhdye, c->X.uhdy1e);
      std::swap(c->X.vhdxe, c->X.vhdx1e);
      std::swap(c->X.hp, c->X.h1p);
    }
    set_views(c, 0);
  } else {
    if (istl == 3) {
      // calpuv9c.f90:282-311 by buffer rotation, UHDY2E <- UHDY1E <- UHDYE and
      // H2P <- H1P <- HP (UHDYE and HP are rewritten for every water cell
      // before they are read), and the copies P1 = P, H1U = HU, H1V = HV
      // (k_advance3)
      xm::DevState &X = c->X;
      double *t = X.uhdy2e;
      X.uhdy2e = X.uhdy1e; X.uhdy1e = X.uhdye; X.uhdye = t;
      t = X.vhdx2e;
      X.vhdx2e = X.vhdx1e; X.vhdx1e = X.vhdxe; X.vhdxe = t;
      t = X.h2p;
      X.h2p = X.h1p; X.h1p = X.hp; X.hp = t;
    }
    set_views(c, istl);
  }
  if (c->device_loops) {
    // the whole step as one graph, its loops on the device
    if (mixed && (rc = choose_inner(c))) return rc;
    StepPlan pl{};
    const xm::Launch lk = c->L();
    pl.mixed = mixed;
    pl.small = !mixed && small_solve(c);
    pl.istl = istl;
    pl.all = all;
    pl.any_isdry = any_isdry;
    pl.any_legacy = any_legacy;
    pl.any99 = any99;
    pl.any_waste = any_waste;
    pl.any_drag = any_drag;
    pl.iters = c->graph_iters;
    pl.max_iterm = 1;
    pl.max_sweeps = 1;
    for (int m = m0; m < m1; ++m) {
      pl.max_iterm = std::max(pl.max_iterm, c->sc_h[m].iterm);
      pl.max_sweeps = std::max(pl.max_sweeps, c->sc_h[m].max_sweeps);
    }
    pl.grid = lk.grid;
    pl.grid_cg = lk.grid_cg;
    pl.grid_cg32 = lk.grid_cg32;
    pl.grid_up32 = lk.grid_up32;
    pl.mx_jac = lk.mx_jac;
    pl.mx_poly = lk.mx_poly;
    pl.may_asym = lk.may_asym;
    pl.chan = lk.chan;
    pl.baro = lk.baro;
    pl.obc_serial = c->obc_serial;
    pl.any_may_asym = c->any_may_asym;
    pl.variant = lk.variant;
    pl.inner_margin = lk.inner_margin;
    pl.ctas_mv = lk.ctas_mv;
    pl.ctas_up = lk.ctas_up;
    pl.nmember = M;
    pl.fac = mixed ? (prm[0].mixed_rsq_factor > 0 ? prm[0].mixed_rsq_factor : 0.1) : 0.0;
    pl.psol = c->psol;
    rc = run_step_graph(c, pl, x_pre, prm, stats, m0, m1);
    if (rc >= 0) {
      if (istl == 0) c->tl3_ready = false;  // CALPUV2C does not keep the three levels
      c->stepped |= m0 == 0 && m1 == M;
      return rc;
    }
    // no graph with conditional nodes here: the host-driven step below
  }
  if (istl == 0) {
    xm::launch_chan_entry(l, c->S, c->X, c->act);
    xm::launch_begin(l, c->S, c->X, c->act, !all);
    if (any_drag) xm::launch_implicit_drag(l, c->S, c->X, c->act);
  } else {
    xm::launch_chan_entry(l, c->S, x_pre, c->act);
    xm::launch_begin3(l, c->S, x_pre, c->act);
    if (any_drag) xm::launch_implicit_drag(l, c->S, x_pre, c->act);
    if (istl == 3) xm::launch_advance3(l, c->S, c->X);
  }
  if (any_isdry) xm::launch_obc_reset(l, c->S, c->B, c->X, c->act);
  CK(cudaGetLastError());
  for (int sweep = 0;; ++sweep) {  // 1000 CONTINUE, for the members still sweeping
    xm::launch_sweep_reset(l, c->ctl, c->act, M);
    xm::launch_assemble(l, c->S, c->X, c->ctl, c->act);
    xm::launch_obc(l, c->S, c->X, c->B, c->ctl, c->act, c->obc_serial, c->any_may_asym ? 1 : 0);
    xm::launch_chan_sub(l, c->S, c->X, c->ctl, c->act, sweep == 0 ? 1 : 0);
    xm::launch_scale(l, c->S, c->X, c->Y, c->ctl, c->act, mixed ? 1 : 0, c->any_may_asym ? 1 : 0);
    CK(cudaGetLastError());
    rc = mixed ? solve_mixed(c, c->X.p, prm[0].mixed_rsq_factor) : solve_fp64(c, c->X.p);
    if (rc) return rc;
    if ((rc = read_glob(c))) return rc;
    if (c->glob_h->err) return device_timeout(c, stats, m0, m1);
    if (c->psol)  // calibration: the adjoint needs P' before P is refreshed from HP
      CK(cudaMemcpyAsync(c->psol, c->X.p, size_t(c->nslot) * sizeof(double),
                         cudaMemcpyDeviceToDevice, c->stream));
    // a member whose solve failed stops here, before the back-substitution
    bool dropped = false;
    int nact = 0;
    for (int m = m0; m < m1; ++m) {
      if (!c->act_h[m]) continue;
      const Ctl &k = c->ctl_h[m];
      efdc_xm_stats &s = stats[m];
      s.iters_last = k.iter;
      s.iters_total += k.iter;
      s.solves += 1;
      s.rsq_last = mixed ? k.rsq64 : k.rsq;
      s.outer_refinements += k.outer;
      s.ccmnm_last = std::min(k.ccmnm_int, k.ccmnm_bc);
      if (k.asym & 2) {
        status[m] = EFDC_XM_UNSUPPORTED;
        set_error("member %d: the scaled operator is unsymmetric although the model has no "
                  "radiation boundary (check SUBO/SVBO next to the open-boundary cells)", m);
      } else if (k.status != EFDC_XM_OK) {
        status[m] = k.status;
        set_error("member %d: CONGRAD: %s after %d iterations (RSQ=%g, RSQM=%g)", m,
                  k.status == EFDC_XM_CG_MAXITER ? "maximum iterations exceeded"
                                                 : "non-finite residual",
                  k.iter, s.rsq_last, prm[m].rsqm);
      }
      if (status[m] != EFDC_XM_OK) {
        c->act_h[m] = 0;
        dropped = true;
      } else {
        ++nact;
      }
    }
    if (nact == 0) break;
    if (dropped && (rc = write_act(c))) return rc;
    xm::launch_chan_flow(l, c->S, c->X, c->act);
    xm::launch_backsub(l, c->S, c->X, c->act);
    xm::launch_obc_hp(l, c->S, c->X, c->B, c->act);
    xm::launch_chan_exch(l, c->S, c->X, c->act);
    bool resweep = false;
    if (any_isdry) {
      xm::launch_wetdry(l, c->S, c->X, c->ctl, c->act, any_legacy, any99);
      CK(cudaGetLastError());
      if ((rc = read_ctl(c))) return rc;
      for (int m = m0; m < m1; ++m) {
        if (!c->act_h[m]) continue;
        const int isd = prm[m].isdry;
        int next = 0;
        if (isd > 0 && isd != 98 && c->ctl_h[m].icordry) {
          if (++ncordry[m] < max_sweeps[m]) {
            next = 1;
          } else {
            status[m] = EFDC_XM_WETDRY_MAXSWEEP;
            set_error("member %d: wet/dry: NCORDRY reached %d", m, max_sweeps[m]);
          }
        }
        c->act_h[m] = next;
        resweep |= next != 0;
      }
    }
    CK(cudaGetLastError());
    if (!resweep) break;
    if ((rc = write_act(c))) return rc;
  }
  // finalisation of the members whose sweeps ended normally
  bool any_fin = false;
  for (int m = m0; m < m1; ++m) {
    c->act_h[m] = (status[m] == EFDC_XM_OK) ? 1 : 0;
    any_fin |= c->act_h[m] != 0;
  }
  if (any_fin) {
    if ((rc = write_act(c))) return rc;
    xm::launch_final(l, c->S, c->X, c->ctl, c->act, any_waste);
    CK(cudaGetLastError());
  }
  if ((rc = read_ctl(c))) return rc;
  if (istl == 0) c->tl3_ready = false;  // CALPUV2C does not keep the three levels
  c->stepped |= m0 == 0 && m1 == M;
  for (int m = m0; m < m1; ++m) {
    efdc_xm_stats &s = stats[m];
    const Ctl &k = c->ctl_h[m];
    s.n_negdep = k.nneg;
    s.n_wasted = k.nwasted;
    if (status[m] == EFDC_XM_OK && k.nnonfinite > 0) {
      status[m] = EFDC_XM_NONFINITE;
      set_error("member %d: non-finite P in %d cells", m, k.nnonfinite);
    }
    if (status[m] == EFDC_XM_OK && k.nneg > 0) status[m] = EFDC_XM_NEG_DEPTH;
    s.status = status[m];
  }
  return overall_status(stats + m0, m1 - m0);
}

// More staging buffers, for transfers in which every array takes its own.
int ensure_stages(efdc_xm_ctx *c, size_t n) {
  while (c->stage.size() < n) {
    double *p = c->alloc<double>(size_t(c->stage_len), false);
    if (!p) {
      set_error("cudaMalloc failed (staging)");
      return EFDC_XM_CUDA_ERROR;
    }
    c->stage.push_back(p);
  }
  return EFDC_XM_OK;
}

// Waits for every stream of the context.
void drain(efdc_xm_ctx *c) {
  for (cudaStream_t s : c->copy_stream) cudaStreamSynchronize(s);
  for (cudaStream_t s : c->dn_stream) cudaStreamSynchronize(s);
  cudaStreamSynchronize(c->up_x);
  cudaStreamSynchronize(c->dn_x);
  cudaStreamSynchronize(c->stream);
}

// Copy streams per direction of a chunked step: each long copy runs at the
// link's speed on one stream, and the copy engines left free serve the other
// direction at the same time.
constexpr int NPIPE = 1;

// efdc_xm_step_batch of a CALPUV2C step in c->nchunk member chunks of about
// equal cell counts, so that the upload of one chunk, the step of an earlier
// one and the download of a still earlier one overlap (the link carries both
// directions at once).  Every array of the two transfers has its own staging
// buffer, in which each member has its own range, so no chunk waits for the
// buffers of another: a chunk's upload (copies on copy_stream, scatter on
// up_x) -> its step (stream) -> its download (gather on dn_x, copies on
// dn_stream), ordered by events.  Results are those of the unchunked call
// bit for bit: every member steps exactly as in a step of all members.
int step_batch_chunks(efdc_xm_ctx *c, const efdc_xm_params *prm, efdc_xm_fields *f,
                      efdc_xm_stats *stats, bool skip_wetdry, bool skip_sbxy) {
  const int M = c->M;
  std::vector<Xfer> up, dn;
  Lists ls;
  uint32_t sent = 0, got = 0;
  int rc = plan_upload(c, f, skip_wetdry, skip_sbxy, false, up, &sent);
  if (rc) {
    fill_status(stats, M, rc);
    return rc;
  }
  {  // the checks see the context as the upload will leave it; a refused call changes nothing
    const bool wd = c->wd_stale, sbxy = c->sbxy_stale, lv = c->tl3_ready;
    const unsigned dr = c->drag_in;
    c->wd_stale = skip_wetdry;
    c->sbxy_stale = skip_sbxy;
    c->tl3_ready = false;
    c->drag_in |= drag_in_of(f);
    rc = validate_step(c, prm, stats);
    c->wd_stale = wd;
    c->sbxy_stale = sbxy;
    c->tl3_ready = lv;
    c->drag_in = dr;
    if (rc) return rc;
  }
  upload_done(c, f, skip_wetdry, skip_sbxy, false);  // the state the step and download see
  const uint32_t sent_before_step = c->synced | sent;
  c->synced = 0;  // until the call has finished (then: what went up or came back)
  if ((rc = plan_download(c, f, skip_wetdry, 0, dn, ls, &got))) {
    fill_status(stats, M, rc);
    return rc;
  }
  const size_t nu = up.size(), nd = dn.size();
  if (nu + nd > size_t(MAX_JOBS)) {
    set_error("internal: too many arrays in one transfer");
    fill_status(stats, M, EFDC_XM_CUDA_ERROR);
    return EFDC_XM_CUDA_ERROR;
  }
  if ((rc = ensure_stages(c, std::max(nu, nd)))) {
    fill_status(stats, M, rc);
    return rc;
  }
  for (size_t j = 0; j < nu; ++j) c->jobs_h[j] = CopyJob{c->stage[j], up[j].dev, up[j].kind};
  for (size_t j = 0; j < nd; ++j) c->jobs_h[nu + j] = CopyJob{c->stage[j], dn[j].dev, dn[j].kind};
  CK(cudaMemcpyAsync(c->jobs_d, c->jobs_h, (nu + nd) * sizeof(CopyJob), cudaMemcpyHostToDevice,
                     c->stream));
  if ((rc = upload_small(c, f))) {  // waits for the solver stream: the job table is in place
    fill_status(stats, M, rc);
    return rc;
  }
  // chunk k holds the members [mb[k], mb[k+1]), about equal cell counts
  const int K = std::min(std::min(c->nchunk, NCHUNK), M);
  std::vector<int> mb(K + 1, M);
  mb[0] = 0;
  {
    long long tot = 0, acc = 0;
    for (int m = 0; m < M; ++m) tot += c->mem[m].la - 1;
    for (int m = 0, k = 1; m < M && k < K; ++m) {
      acc += c->mem[m].la - 1;
      if (acc * K >= tot * k) mb[k++] = m + 1;
    }
  }
  auto slots = [&](int k, int &d0, int &d1) {  // the members' ghost tiles included
    d0 = (c->mem[mb[k]].tile0 - 1) * xm::TILE;
    d1 = c->mem[mb[k + 1] - 1].tile1 * xm::TILE;
  };
  // the transfer streams start after the solver stream's earlier work
  CK(cudaEventRecord(c->ev_start, c->stream));
  for (cudaStream_t s : c->copy_stream) CK(cudaStreamWaitEvent(s, c->ev_start, 0));
  for (cudaStream_t s : c->dn_stream) CK(cudaStreamWaitEvent(s, c->ev_start, 0));
  CK(cudaStreamWaitEvent(c->up_x, c->ev_start, 0));
  CK(cudaStreamWaitEvent(c->dn_x, c->ev_start, 0));
  int q = 0, d0 = 0, d1 = 0;
  for (int k = 0; k < K; ++k) {  // all uploads, queued
    if (mb[k] == mb[k + 1]) continue;
    for (size_t j = 0; j < nu; ++j)
      if ((rc = h2d_range(c, up[j], reinterpret_cast<char *>(c->stage[j]), mb[k], mb[k + 1],
                          c->copy_stream, q, NPIPE))) {
        drain(c);
        return rc;
      }
    for (int s = 0; s < NPIPE; ++s) {
      CK(cudaEventRecord(c->ev_j[k][s], c->copy_stream[s]));
      CK(cudaStreamWaitEvent(c->up_x, c->ev_j[k][s], 0));
    }
    slots(k, d0, d1);
    xm::launch_scatter(c->up_x, c->jobs_d, int(nu), c->lidx, c->tile_member, c->moff, c->mlc, d0,
                       d1);
    CK(cudaGetLastError());
    if ((rc = copy_levels(c, f, size_t(d0), size_t(d1), c->up_x))) {
      drain(c);
      return rc;
    }
    CK(cudaEventRecord(c->ev_up[k], c->up_x));
  }
  std::vector<Keep> keep;
  auto fail = [&](int r) {  // the copies queued so far end; the caller's kept elements return
    drain(c);
    for (const Keep &kp : keep) std::memcpy(kp.at, kp.val, kp.n);
    return r;
  };
  const bool recip = f[0].hpi || f[0].hui || f[0].hvi;
  q = 0;
  struct Flag {  // c->in_chunks for the steps below, on every way out
    bool &f;
    explicit Flag(bool &x) : f(x) { f = true; }
    ~Flag() { f = false; }
  } in_chunks(c->in_chunks);
  for (int k = 0; k < K; ++k) {  // steps, each followed by its download, queued
    if (mb[k] == mb[k + 1]) continue;
    CK(cudaStreamWaitEvent(c->stream, c->ev_up[k], 0));
    rc = step_range(c, prm, stats, mb[k], mb[k + 1]);
    if (rc == EFDC_XM_CUDA_ERROR || rc == EFDC_XM_BAD_ARGUMENT) return fail(rc);
    if (recip)  // 1/HP, 1/HU, 1/HV are formed on request
      xm::launch_reciprocals(c->L(), c->S, c->X, c->mem[mb[k]].tile0,
                             c->mem[mb[k + 1] - 1].tile1);
    CK(cudaEventRecord(c->ev_step[k], c->stream));
    CK(cudaStreamWaitEvent(c->dn_x, c->ev_step[k], 0));
    slots(k, d0, d1);
    xm::launch_gather(c->dn_x, c->jobs_d + nu, int(nd), c->lidx, c->tile_member, c->moff, d0, d1);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->ev_g[k], c->dn_x));
    for (int s = 0; s < NPIPE; ++s) CK(cudaStreamWaitEvent(c->dn_stream[s], c->ev_g[k], 0));
    for (size_t j = 0; j < nd; ++j)
      if ((rc = d2h_range(c, dn[j], reinterpret_cast<const char *>(c->stage[j]), mb[k],
                          mb[k + 1], c->dn_stream, q, keep, NPIPE)))
        return fail(rc);
  }
  fail(0);
  CK(cudaGetLastError());
  if ((rc = download_finish(c, f, ls))) return rc;
  // the kept copies, those that went up and were not written by the steps,
  // and those that came back
  c->synced = (sent_before_step & ~(skip_wetdry ? STEP_WRITES_DRYFREE : STEP_WRITES)) | got;
  c->stepped = true;  // the chunks together stepped every member
  return overall_status(stats, M);
}

// LAWET, LADRY of the members whose lists were asked for (calpuv2c.f90:1061-1080).
int batch_lists_stats(const efdc_xm_ctx *c, const efdc_xm_params *prm, const efdc_xm_fields *f,
                      efdc_xm_stats *stats, int st) {
  for (int m = 0; m < c->M; ++m) {
    if (!(f[m].lwet || f[m].ldry)) continue;
    const Member &mb = c->mem[m];
    if (prm[m].isdry == 0) {
      stats[m].lawet = mb.la - 1;
      stats[m].ladry = 0;
    } else {
      int nw = 0, nd = 0;
      for (int L = 2; L <= mb.la; ++L) {
        if (f[m].lmaskdry[L - 1]) ++nw;
        else if ((!mb.oldmask_h.empty() && mb.oldmask_h[L - 1]) || prm[m].n < prm[m].ntstbc + 1)
          ++nd;
      }
      stats[m].lawet = nw;
      stats[m].ladry = nd;
    }
  }
  return st;
}
}  // namespace

extern "C" {

int32_t efdc_xm_step_device_batch(efdc_xm_ctx *c, const efdc_xm_params *prm,
                                  efdc_xm_stats *stats) {
  if (!c || !prm || !stats) {
    set_error("efdc_xm_step_device: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  std::memset(stats, 0, sizeof(efdc_xm_stats) * c->M);
  const int rc = validate_step(c, prm, stats);
  if (rc) return rc;
  return step_range(c, prm, stats, 0, c->M);
}


int32_t efdc_xm_step_batch(efdc_xm_ctx *c, const efdc_xm_params *prm, efdc_xm_fields *f,
                           efdc_xm_stats *stats) {
  if (!c || !prm || !f || !stats) {
    set_error("efdc_xm_step: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  const int M = c->M;
  std::memset(stats, 0, sizeof(efdc_xm_stats) * M);
  for (int m = 0; m < M; ++m) {
    const efdc_xm_fields &x = f[m];
    if (!x.p || !x.hp || !x.hu || !x.hv || !x.uhdye || !x.vhdxe || !x.sub || !x.svb) {
      set_error("efdc_xm_step: member %d: NULL argument (P, HP, HU, HV, UHDYE, VHDXE, SUB, SVB "
                "are required)", m);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
    if (prm[m].bsc > 1.E-6 && !x.b) {
      set_error("efdc_xm_step: member %d: BSC > 1E-6 needs B", m);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
    if (prm[m].isdry > 0 && (!x.sbx || !x.sby || !x.lmaskdry || !x.iscdry)) {
      set_error("efdc_xm_step: member %d: ISDRY>0 needs SBX, SBY, LMASKDRY and ISCDRY", m);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
    if (prm[m].tl3_istl != 0 && prm[m].bsc > 1.E-6 && (!x.fpgxe || !x.fpgye)) {
      set_error("efdc_xm_step: member %d: CALPUV9C with BSC > 1E-6 needs FPGXE and FPGYE", m);
      fill_status(stats, M, EFDC_XM_BAD_ARGUMENT);
      return EFDC_XM_BAD_ARGUMENT;
    }
  }
  const int istl = prm[0].tl3_istl;
  bool no_wetdry = true, no_baro = true;
  for (int m = 0; m < M; ++m) {
    no_wetdry &= prm[m].isdry == 0;
    no_baro &= !(prm[m].bsc > 1.E-6);
  }
  if (istl == 0 && M >= 2 && !wants_system(f) && !c->calib) {
    const int st = step_batch_chunks(c, prm, f, stats, no_wetdry, no_wetdry && no_baro);
    if (st == EFDC_XM_CUDA_ERROR || st == EFDC_XM_BAD_ARGUMENT) return st;
    return batch_lists_stats(c, prm, f, stats, st);
  }
  int rc = upload_batch(c, f, no_wetdry, no_wetdry && no_baro, istl != 0);
  if (rc) {
    fill_status(stats, M, rc);
    return rc;
  }
  const int st = efdc_xm_step_device_batch(c, prm, stats);
  if (st == EFDC_XM_CUDA_ERROR || st == EFDC_XM_BAD_ARGUMENT) return st;
  if ((rc = download_batch(c, f, no_wetdry, istl))) {
    fill_status(stats, M, rc);
    return rc;
  }
  return batch_lists_stats(c, prm, f, stats, st);
}

}  // extern "C"

namespace {
int single_only(const efdc_xm_ctx *c, const char *who) {
  if (!c) {
    set_error("%s: NULL context", who);
    return EFDC_XM_BAD_ARGUMENT;
  }
  if (c->M != 1) {
    set_error("%s: the context holds %d members; use the _batch entry point", who, c->M);
    return EFDC_XM_BAD_ARGUMENT;
  }
  return EFDC_XM_OK;
}
}  // namespace

extern "C" {

// ---- single-basin entry points: the batch API with one member ----
int32_t efdc_xm_upload(efdc_xm_ctx *c, const efdc_xm_fields *f) {
  const int rc = single_only(c, "efdc_xm_upload");
  return rc ? rc : efdc_xm_upload_batch(c, f);
}

int32_t efdc_xm_download(efdc_xm_ctx *c, efdc_xm_fields *f) {
  const int rc = single_only(c, "efdc_xm_download");
  return rc ? rc : efdc_xm_download_batch(c, f);
}

int32_t efdc_xm_step_device(efdc_xm_ctx *c, const efdc_xm_params *prm, efdc_xm_stats *stats) {
  efdc_xm_stats dummy;
  if (!stats) stats = &dummy;
  std::memset(stats, 0, sizeof(*stats));
  const int rc = single_only(c, "efdc_xm_step_device");
  if (rc) return stats->status = rc;
  return efdc_xm_step_device_batch(c, prm, stats);
}

int32_t efdc_xm_step(efdc_xm_ctx *c, const efdc_xm_params *prm, efdc_xm_fields *f,
                     efdc_xm_stats *stats) {
  efdc_xm_stats dummy;
  if (!stats) stats = &dummy;
  std::memset(stats, 0, sizeof(*stats));
  const int rc = single_only(c, "efdc_xm_step");
  if (rc) return stats->status = rc;
  return efdc_xm_step_batch(c, prm, f, stats);
}

namespace {
// CUDA graphs hold the kernels' arguments; a change of the channel arrays
// drops them (they are captured again on next use).
void drop_graphs(efdc_xm_ctx *c) {
  for (cudaGraphExec_t &g : c->graph_cg)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  for (cudaGraphExec_t &g : c->graph_mx)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  for (bool &f : c->graph_cg_failed) f = false;
  for (bool &f : c->graph_mx_failed) f = false;
  drop_step_graphs(c);
}

// S.ch from every member's channel list, and the slot kinds (channel cells
// are CHAN).  Channels are few: plain host-side packing and small copies.
int rebuild_channels(efdc_xm_ctx *c) {
  CK(cudaStreamSynchronize(c->stream));
  for (void *b : c->chan_bufs) cudaFree(b);
  c->chan_bufs.clear();
  xm::DevChan &C = c->S.ch;
  C = xm::DevChan{};
  c->chan_hp1 = nullptr;
  const int M = c->M;
  std::vector<uint8_t> kind = c->kind_h;
  std::vector<int> cstart(M + 1, 0), type, host, guest, gu, qh, qg, fh, fg;
  std::vector<double> len, fric, gw, gl;
  for (int m = 0; m < M; ++m) {
    cstart[m] = int(type.size());
    const Member &mb = c->mem[m];
    std::vector<int> seen;
    auto first = [&](int d) {
      if (std::find(seen.begin(), seen.end(), d) != seen.end()) return 0;
      seen.push_back(d);
      return 1;
    };
    auto quad = [&](int d) { return c->qstart_h[m] + (d / xm::TILE - mb.tile0) / 4; };
    for (const ChanSpec &k : c->chans[m]) {
      const int dh = mb.slot_of[k.lh], dg = mb.slot_of[k.type == 1 ? k.lu : k.lv];
      type.push_back(k.type);
      host.push_back(dh);
      guest.push_back(dg);
      gu.push_back(k.type == 2 && k.lu >= 2 ? mb.slot_of[k.lu] : -1);
      qh.push_back(quad(dh));
      qg.push_back(quad(dg));
      fg.push_back(first(dg));
      fh.push_back(first(dh));
      len.push_back(k.len);
      fric.push_back(k.fric);
      gw.push_back(k.gw);
      gl.push_back(k.gl);
      kind[dh] = kind[dg] = xm::CHAN;
    }
  }
  const int n = int(type.size());
  cstart[M] = n;
  c->chan_start = cstart;
  CK(cudaMemcpy(const_cast<uint8_t *>(c->S.kind), kind.data(), kind.size(), cudaMemcpyHostToDevice));
  drop_graphs(c);
  if (n == 0) {
    CK(cudaDeviceSynchronize());  // the kinds are in place before the next launch
    return EFDC_XM_OK;
  }
  auto dev = [&](const void *src, size_t bytes) -> void * {
    void *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 1)) != cudaSuccess) return nullptr;
    c->chan_bufs.push_back(p);
    if (src)
      cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
    else
      cudaMemset(p, 0, bytes);
    return p;
  };
  const size_t ni = sizeof(int) * size_t(n), nd = sizeof(double) * size_t(n);
  C.cstart = static_cast<const int *>(dev(cstart.data(), sizeof(int) * (M + 1)));
  C.type = static_cast<const int *>(dev(type.data(), ni));
  C.host = static_cast<const int *>(dev(host.data(), ni));
  C.guest = static_cast<const int *>(dev(guest.data(), ni));
  C.gu = static_cast<const int *>(dev(gu.data(), ni));
  C.qhost = static_cast<const int *>(dev(qh.data(), ni));
  C.qguest = static_cast<const int *>(dev(qg.data(), ni));
  C.first_host = static_cast<const int *>(dev(fh.data(), ni));
  C.first_guest = static_cast<const int *>(dev(fg.data(), ni));
  C.len = static_cast<const double *>(dev(len.data(), nd));
  C.fric = static_cast<const double *>(dev(fric.data(), nd));
  C.gw = static_cast<const double *>(dev(gw.data(), nd));
  C.gl = static_cast<const double *>(dev(gl.data(), nd));
  c->chan_hp1 = static_cast<double *>(dev(c->hp1_h.data(), sizeof(double) * M));
  C.hp1 = c->chan_hp1;
  double **st[] = {&C.qu, &C.qv, &C.qun, &C.qvn, &C.qut, &C.qvt, &C.cu,
                   &C.cv, &C.chh, &C.p1h, &C.p1g, &C.p0h, &C.p0g};
  for (double **q : st) *q = static_cast<double *>(dev(nullptr, nd));
  C.hh32 = static_cast<float *>(dev(nullptr, sizeof(float) * size_t(n)));
  C.iact = static_cast<int *>(dev(nullptr, ni));
  for (void *b : c->chan_bufs)
    if (!b) {
      set_error("efdc_xm_set_channels: device allocation failed");
      return EFDC_XM_CUDA_ERROR;
    }
  if (c->chan_bufs.size() != 29) {
    set_error("internal: channel arrays");
    return EFDC_XM_CUDA_ERROR;
  }
  // copies and zeroing ran on the legacy stream, which the context's stream
  // does not wait for
  CK(cudaDeviceSynchronize());
  C.n = n;
  return EFDC_XM_OK;
}
}  // namespace

int32_t efdc_xm_set_layers(efdc_xm_ctx *c, int32_t member, const efdc_xm_layers *ly) {
  if (!c || !ly || member < 0 || member >= c->M || ly->kc < 1 || ly->kc > 64 || !ly->dzc ||
      !ly->zz || ly->ld < c->mem[member].lc) {
    set_error("efdc_xm_set_layers: need a context, a member, 1 <= kc <= 64, ld >= LC and the "
              "DZC, ZZ arrays");
    return EFDC_XM_BAD_ARGUMENT;
  }
  xm::DevBaro &Bc = c->S.baro;
  if (Bc.kc != 0 && Bc.kc != ly->kc) {
    set_error("efdc_xm_set_layers: the members of a context share KC (%d, not %d)", Bc.kc,
              ly->kc);
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  const size_t ns = c->nslot;
  if (Bc.kc == 0) {  // the planes, once (zeroed: land slots stay 0)
    double *dzc = c->alloc<double>(ns * ly->kc), *zz = c->alloc<double>(ns * ly->kc);
    double *b = c->alloc<double>(ns * ly->kc);
    double *bi1 = c->alloc<double>(ns), *bi2 = c->alloc<double>(ns), *be = c->alloc<double>(ns);
    if (!dzc || !zz || !b || !bi1 || !bi2 || !be) {
      set_error("efdc_xm_set_layers: device allocation failed");
      return EFDC_XM_CUDA_ERROR;
    }
    Bc.dzc = dzc;
    Bc.zz = zz;
    Bc.b = b;
    Bc.bi1 = bi1;
    Bc.bi2 = bi2;
    Bc.be = be;
    Bc.stride = (long long)ns;
    Bc.kc = ly->kc;
    int lcmax = 0;
    for (const Member &mb : c->mem) lcmax = std::max(lcmax, mb.lc);
    c->zeros_h.assign(size_t(lcmax) + 1, 0.0);
  }
  // the member's cells of each layer, host order -> tile order
  const Member &mb = c->mem[member];
  const int n = mb.la - 1;
  std::vector<int> idx(n);
  for (int L = 2; L <= mb.la; ++L) idx[L - 2] = mb.slot_of[L];
  std::vector<double> val(size_t(n) * 2 * ly->kc);
  for (int k = 0; k < ly->kc; ++k)
    for (int L = 2; L <= mb.la; ++L) {
      val[(size_t(2 * k)) * n + (L - 2)] = ly->dzc[size_t(k) * ly->ld + (L - 1)];
      val[(size_t(2 * k + 1)) * n + (L - 2)] = ly->zz[size_t(k) * ly->ld + (L - 1)];
    }
  int *idx_d = nullptr;
  double *val_d = nullptr;
  if (cudaMalloc(&idx_d, sizeof(int) * std::max(n, 1)) != cudaSuccess ||
      cudaMalloc(&val_d, sizeof(double) * std::max<size_t>(val.size(), 1)) != cudaSuccess) {
    cudaFree(idx_d);
    set_error("efdc_xm_set_layers: device allocation failed");
    return EFDC_XM_CUDA_ERROR;
  }
  // the context's stream does not wait for the legacy stream: the zeroing of
  // new planes and these copies must be complete before the scatter runs
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpyAsync(idx_d, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(val_d, val.data(), sizeof(double) * val.size(), cudaMemcpyHostToDevice,
                      c->stream) != cudaSuccess) {
    cudaFree(idx_d);
    cudaFree(val_d);
    set_error("efdc_xm_set_layers: copy failed");
    return EFDC_XM_CUDA_ERROR;
  }
  for (int k = 0; k < ly->kc; ++k) {
    xm::launch_put(c->stream, idx_d, val_d + size_t(2 * k) * n, n,
                   const_cast<double *>(Bc.dzc) + size_t(k) * ns);
    xm::launch_put(c->stream, idx_d, val_d + size_t(2 * k + 1) * n, n,
                   const_cast<double *>(Bc.zz) + size_t(k) * ns);
  }
  const cudaError_t e = cudaStreamSynchronize(c->stream);
  cudaFree(idx_d);
  cudaFree(val_d);
  if (e != cudaSuccess) {
    set_error("efdc_xm_set_layers: %s", cudaGetErrorString(e));
    return EFDC_XM_CUDA_ERROR;
  }
  c->has_layers[member] = 1;
  drop_graphs(c);  // the kernels' static views (the layer arrays) have changed
  return EFDC_XM_OK;
}

int32_t efdc_xm_set_bed(efdc_xm_ctx *c, int32_t member, const efdc_xm_bed *bed) {
  if (!c || !bed || member < 0 || member >= c->M || !bed->zbr || !bed->stbxo || !bed->stbyo ||
      !bed->dxp || !bed->dyp || !bed->dzc1 || !bed->sgzu1 || !bed->sgzv1 || bed->kc < 1) {
    set_error("efdc_xm_set_bed: need a context, a member, KC >= 1 and the ZBR, STBXO, STBYO, "
              "DXP, DYP, DZC1, SGZU1, SGZV1 arrays");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  xm::DevBed &Bd = c->bed;
  if (!c->bed_alloc) {  // zeroed: STBX, STBY start at 0 (caltbxy.f90:112-116)
    double *b[15];
    for (double *&p : b)
      if (!(p = c->alloc<double>(size_t(c->nslot)))) {
        set_error("efdc_xm_set_bed: device allocation failed");
        return EFDC_XM_CUDA_ERROR;
      }
    c->ds = c->alloc<xm::DragScalars>(size_t(c->M));
    if (!c->ds) {
      set_error("efdc_xm_set_bed: device allocation failed");
      return EFDC_XM_CUDA_ERROR;
    }
    Bd.zbr = b[0]; Bd.zbratu = b[1]; Bd.zbratv = b[2]; Bd.sgzuu = b[3]; Bd.sgzvv = b[4];
    Bd.stbxo = b[5]; Bd.stbyo = b[6]; Bd.stbx = b[7]; Bd.stby = b[8];
    Bd.ub = b[9]; Bd.vb = b[10]; Bd.vu = b[11]; Bd.uv = b[12]; Bd.h1u = b[13]; Bd.h1v = b[14];
    c->has_bed.assign(c->M, 0);
    c->bed_sc.assign(c->M, xm::DragScalars{});
    CK(cudaDeviceSynchronize());  // the zeroing ran on the legacy stream
    c->bed_alloc = true;
  }
  // the member's arrays into tile order (its slots; tile 0, the ghost tile,
  // with member 0); DXP, DYP, DZC1, SGZU1, SGZV1 pass through the per-call
  // input buffers, free here
  const int M = c->M;
  auto one = [&](const double *a) {
    std::vector<const void *> v(M, nullptr);
    v[member] = a;
    return v;
  };
  const std::vector<Xfer> xs = {
      Xfer{one(bed->zbr), const_cast<double *>(Bd.zbr), 0},
      Xfer{one(bed->stbxo), const_cast<double *>(Bd.stbxo), 0},
      Xfer{one(bed->stbyo), const_cast<double *>(Bd.stbyo), 0},
      Xfer{one(bed->dxp), Bd.ub, 0},   Xfer{one(bed->dyp), Bd.vb, 0},
      Xfer{one(bed->dzc1), Bd.vu, 0},  Xfer{one(bed->sgzu1), Bd.uv, 0},
      Xfer{one(bed->sgzv1), Bd.h1u, 0}};
  if (xs.size() > size_t(NSTAGE)) {
    set_error("internal: too many bed arrays");
    return EFDC_XM_CUDA_ERROR;
  }
  for (size_t j = 0; j < xs.size(); ++j)
    c->jobs_h[j] = CopyJob{c->stage[j], xs[j].dev, xs[j].kind};
  CK(cudaMemcpyAsync(c->jobs_d, c->jobs_h, xs.size() * sizeof(CopyJob), cudaMemcpyHostToDevice,
                     c->stream));
  int rc = copies_after_compute(c), k = 0;
  for (size_t j = 0; !rc && j < xs.size(); ++j)
    rc = h2d_range(c, xs[j], reinterpret_cast<char *>(c->stage[j]), member, member + 1,
                   c->copy_stream, k);
  if (!rc) rc = compute_after_copies(c);
  if (rc) return rc;
  const Member &mb = c->mem[member];
  const int d0 = (mb.tile0 - 1) * xm::TILE, d1 = mb.tile1 * xm::TILE;  // with its ghost tile
  xm::launch_scatter(c->stream, c->jobs_d, int(xs.size()), c->lidx, c->tile_member, c->moff,
                     c->mlc, d0, d1);
  const size_t g = size_t(mb.lc) - 1;  // the ghost cell LC
  xm::launch_bed(c->stream, c->S, Bd, Bd.ub, Bd.vb, Bd.vu, Bd.uv, Bd.h1u,
                 bed->dxp[g] * bed->zbr[g], bed->dyp[g] * bed->zbr[g], mb.tile0, mb.tile1);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  xm::DragScalars &q = c->bed_sc[member];
  q.avcon = bed->avcon;
  q.vismud = bed->vismud;
  q.visfac = 0.0258 * std::pow(bed->coeftsbl, 2. / 7.);  // caltbxy.f90:210-211
  q.kc1 = bed->kc == 1 ? 1 : 0;
  c->has_bed[member] = 1;
  return EFDC_XM_OK;
}

int32_t efdc_xm_bottom_stress_batch(efdc_xm_ctx *c, const efdc_xm_drag_params *prm,
                                    efdc_xm_drag_fields *f) {
  if (!c || !prm || !f) {
    set_error("efdc_xm_bottom_stress: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  c->synced &= ~uint32_t(EFDC_XM_SAME_TBX | EFDC_XM_SAME_TBY);  // written on the device
  const int M = c->M;
  for (int m = 0; m < M; ++m) {
    const efdc_xm_drag_fields &x = f[m];
    if (!c->bed_alloc || !c->has_bed[m] || !(prm[m].delt > 0) || !x.ub || !x.vb || !x.vu ||
        !x.uv || !x.h1u || !x.h1v) {
      set_error("efdc_xm_bottom_stress: member %d: needs its bed (efdc_xm_set_bed), DELT > 0 "
                "and the UB, VB, VU, UV, H1U, H1V arrays", m);
      return EFDC_XM_BAD_ARGUMENT;
    }
    if (prm[m].isdry > 0 && c->wd_stale) {
      set_error("efdc_xm_bottom_stress: member %d has ISDRY > 0 but the device's LMASKDRY was "
                "left on the host by a step without wetting and drying: upload it first", m);
      return EFDC_XM_BAD_ARGUMENT;
    }
  }
  CK(cudaSetDevice(c->device));
  xm::DevBed &Bd = c->bed;
  std::vector<Xfer> up, dn;
  auto per = [&](const double *efdc_xm_drag_fields::*a) {
    std::vector<const void *> v(M);
    for (int m = 0; m < M; ++m) v[m] = f[m].*a;
    return v;
  };
  up.push_back(Xfer{per(&efdc_xm_drag_fields::ub), Bd.ub, 0});
  up.push_back(Xfer{per(&efdc_xm_drag_fields::vb), Bd.vb, 0});
  up.push_back(Xfer{per(&efdc_xm_drag_fields::vu), Bd.vu, 0});
  up.push_back(Xfer{per(&efdc_xm_drag_fields::uv), Bd.uv, 0});
  up.push_back(Xfer{per(&efdc_xm_drag_fields::h1u), Bd.h1u, 0});
  up.push_back(Xfer{per(&efdc_xm_drag_fields::h1v), Bd.h1v, 0});
  int rc = upload_arrays(c, up);
  if (rc) return rc;
  for (int m = 0; m < M; ++m) {
    xm::DragScalars q = c->bed_sc[m];
    q.delt = prm[m].delt;
    q.avcon1 = prm[m].avcon1;
    q.isdry = prm[m].isdry;
    q.n = prm[m].n;
    q.ntstbc = prm[m].ntstbc;
    q.on = 1;
    c->bed_sc[m] = q;
  }
  CK(cudaMemcpyAsync(c->ds, c->bed_sc.data(), sizeof(xm::DragScalars) * M,
                     cudaMemcpyHostToDevice, c->stream));
  xm::launch_tbxy(c->L(), c->S, c->X, Bd, c->ds);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));  // the host copy of the scalars may change after this
  rc = 0;
#define XM_DN(name, dev)                                                        \
  {                                                                             \
    std::vector<const void *> v(M);                                             \
    for (int m = 0; m < M; ++m) v[m] = f[m].name;                               \
    if ((rc = collect(c, dn, v, dev, 0, #name))) return rc;                     \
  }
  XM_DN(stbx, Bd.stbx) XM_DN(stby, Bd.stby) XM_DN(tbx, c->X.tbx) XM_DN(tby, c->X.tby)
#undef XM_DN
  return download_arrays(c, dn);
}

// Arrays of one member into tile order: its slots and its ghost tile (which
// takes element LC), NSTAGE arrays per round through the staging buffers.
int upload_member(efdc_xm_ctx *c, int member, const std::vector<Xfer> &xs) {
  const Member &mb = c->mem[member];
  const int d0 = (mb.tile0 - 1) * xm::TILE, d1 = mb.tile1 * xm::TILE;
  for (size_t g0 = 0; g0 < xs.size(); g0 += NSTAGE) {
    const size_t g1 = std::min(xs.size(), g0 + NSTAGE);
    for (size_t j = g0; j < g1; ++j)
      c->jobs_h[j - g0] = CopyJob{c->stage[j - g0], xs[j].dev, xs[j].kind};
    CK(cudaMemcpyAsync(c->jobs_d, c->jobs_h, (g1 - g0) * sizeof(CopyJob),
                       cudaMemcpyHostToDevice, c->stream));
    int rc = copies_after_compute(c), k = 0;
    for (size_t j = g0; !rc && j < g1; ++j)
      rc = h2d_range(c, xs[j], reinterpret_cast<char *>(c->stage[j - g0]), member, member + 1,
                     c->copy_stream, k);
    if (!rc) rc = compute_after_copies(c);
    if (rc) return rc;
    xm::launch_scatter(c->stream, c->jobs_d, int(g1 - g0), c->lidx, c->tile_member, c->moff,
                       c->mlc, d0, d1);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));  // the staging buffers and jobs are reused
  }
  return EFDC_XM_OK;
}

// Per-layer arrays as transfers: layer k of member m at host[m] + k*ld[m].
void layer_xfers(std::vector<Xfer> &out, const std::vector<const double *> &host,
                 const std::vector<int> &ld, double *dev, size_t ls, int kc) {
  for (int k = 0; k < kc; ++k) {
    std::vector<const void *> v(host.size());
    for (size_t m = 0; m < host.size(); ++m)
      v[m] = host[m] ? static_cast<const void *>(host[m] + size_t(k) * ld[m]) : nullptr;
    out.push_back(Xfer{v, dev + size_t(k) * ls, 0});
  }
}

int32_t efdc_xm_set_momentum(efdc_xm_ctx *c, int32_t member, const efdc_xm_momentum *mo) {
  if (!c || !mo || member < 0 || member >= c->M) {
    set_error("efdc_xm_set_momentum: need a context, a member index and the static part");
    return EFDC_XM_BAD_ARGUMENT;
  }
  const Member &mb = c->mem[member];
  if (mo->kc < 1 || mo->kc > 64 || mo->ld < mb.lc || !mo->fcorc || !mo->dydi || !mo->dxdj ||
      !mo->scax || !mo->scay || !mo->saax || !mo->saay || !mo->sgzu || !mo->sgzv || !mo->fsgzu ||
      !mo->fsgzv || !mo->lnwc || !mo->lsec || mo->nbcs < 0 ||
      (mo->nbcs > 0 && (!mo->lbcs || !mo->lberc || !mo->lbnrc)) || (!mo->sdx != !mo->sdy) ||
      (mo->sdx && !mo->lhdmf)) {
    set_error("efdc_xm_set_momentum: member %d: need 1 <= KC <= 64, LD >= LC, FCORC, DYDI, "
              "DXDJ, SCAX, SCAY, SAAX, SAAY, the SGZU, SGZV, FSGZU, FSGZV layers, LNWC, LSEC, "
              "the NBCS boundary lists, and SDX with SDY and LHDMF or none", member);
    return EFDC_XM_BAD_ARGUMENT;
  }
  if (c->mom_alloc && mo->kc > c->mom_kc) {
    set_error("efdc_xm_set_momentum: member %d has KC = %d, more than the %d layers of the "
              "context's first member with momentum", member, mo->kc, c->mom_kc);
    return EFDC_XM_BAD_ARGUMENT;
  }
  for (const int32_t *a : {mo->lnwc, mo->lsec})
    for (int L = 2; L <= mb.la; ++L)
      if (a[L - 1] < 1 || a[L - 1] > mb.lc) {
        set_error("efdc_xm_set_momentum: member %d: LNWC/LSEC(%d) = %d is outside 1..LC", member,
                  L, a[L - 1]);
        return EFDC_XM_BAD_ARGUMENT;
      }
  for (int j = 0; j < mo->nbcs; ++j)
    for (const int32_t *a : {mo->lbcs, mo->lberc, mo->lbnrc})
      if (a[j] > mb.lc) {
        set_error("efdc_xm_set_momentum: member %d: a boundary list entry %d exceeds LC", member,
                  a[j]);
        return EFDC_XM_BAD_ARGUMENT;
      }
  CK(cudaSetDevice(c->device));
  const int M = c->M;
  const size_t ns = size_t(c->nslot);
  xm::MomDev &D = c->md;
  if (!c->mom_alloc) {  // zeroed: land slots and cells outside the wet set stay 0
    const int kc = mo->kc;
    c->mom_kc = kc;
    auto A = [&](size_t n) { return c->alloc<double>(n); };
    double *st[10];
    for (double *&q : st) q = A(ns);
    int *in[4];
    for (int *&q : in) q = c->alloc<int>(ns);
    double *ly[23];
    for (double *&q : ly) q = A(ns * kc);
    c->mom_hp = A(ns);
    D.cacsum = A(size_t(M));
    xm::MomScalars *sc = c->alloc<xm::MomScalars>(size_t(M));
    for (double *q : st) if (!q) sc = nullptr;
    for (int *q : in) if (!q) sc = nullptr;
    for (double *q : ly) if (!q) sc = nullptr;
    if (!sc || !c->mom_hp || !D.cacsum) {
      set_error("efdc_xm_set_momentum: device allocation failed (%d layers)", kc);
      return EFDC_XM_CUDA_ERROR;
    }
    D.fcorc = st[0]; D.dydi = st[1]; D.dxdj = st[2]; D.scax = st[3]; D.scay = st[4];
    D.saax = st[5]; D.saay = st[6]; D.stcuv = st[7]; D.sdx = st[8]; D.sdy = st[9];
    D.lhdmf = in[0]; D.nw = in[1]; D.se = in[2]; D.wet = in[3];
    D.sgzu = ly[0]; D.sgzv = ly[1]; D.fsgzu = ly[2]; D.fsgzv = ly[3];
    D.u = ly[4]; D.v = ly[5]; D.uhdy = ly[6]; D.vhdx = ly[7]; D.fuhj = ly[8]; D.fvhj = ly[9];
    D.fmdux = ly[10]; D.fmduy = ly[11]; D.fmdvx = ly[12]; D.fmdvy = ly[13];
    D.fuhu = ly[14]; D.fvhu = ly[15]; D.fvhv = ly[16]; D.fuhv = ly[17]; D.cac = ly[18];
    D.fcax = ly[19]; D.fcay = ly[20]; D.fx = ly[21]; D.fy = ly[22];
    D.sc = sc;
    D.ls = ns;
    c->has_mom.assign(M, 0);
    c->mom_ld.assign(M, 0);
    c->mom_t2.assign(M, {});
    c->mom_bc.assign(M, {});
    c->mom_sc_h.assign(M, xm::MomScalars{});
    CK(cudaDeviceSynchronize());  // the zeroing ran on the legacy stream
    c->mom_alloc = true;
  }
  const int kc = mo->kc;
  auto one = [&](const void *a) {
    std::vector<const void *> v(M, nullptr);
    v[member] = a;
    return v;
  };
  std::vector<Xfer> xs = {
      Xfer{one(mo->fcorc), const_cast<double *>(D.fcorc), 0},
      Xfer{one(mo->dydi), const_cast<double *>(D.dydi), 0},
      Xfer{one(mo->dxdj), const_cast<double *>(D.dxdj), 0},
      Xfer{one(mo->scax), const_cast<double *>(D.scax), 0},
      Xfer{one(mo->scay), const_cast<double *>(D.scay), 0},
      Xfer{one(mo->saax), const_cast<double *>(D.saax), 0},
      Xfer{one(mo->saay), const_cast<double *>(D.saay), 0}};
  if (mo->stcuv) xs.push_back(Xfer{one(mo->stcuv), const_cast<double *>(D.stcuv), 0});
  if (mo->sdx) {
    xs.push_back(Xfer{one(mo->sdx), const_cast<double *>(D.sdx), 0});
    xs.push_back(Xfer{one(mo->sdy), const_cast<double *>(D.sdy), 0});
    xs.push_back(Xfer{one(mo->lhdmf), const_cast<int *>(D.lhdmf), 1});
  }
  std::vector<const double *> h(M, nullptr);
  std::vector<int> ld(M, 0);
  ld[member] = mo->ld;
  const double *const lay[4] = {mo->sgzu, mo->sgzv, mo->fsgzu, mo->fsgzv};
  const double *const dl[4] = {D.sgzu, D.sgzv, D.fsgzu, D.fsgzv};
  for (int a = 0; a < 4; ++a) {
    h[member] = lay[a];
    layer_xfers(xs, h, ld, const_cast<double *>(dl[a]), D.ls, kc);
  }
  int rc = upload_member(c, member, xs);
  if (rc) return rc;
  // the diagonal neighbours' slots (LC: the member's ghost slot)
  auto slot = [&](int L) { return (L >= 2 && L <= mb.la) ? mb.slot_of[L] : (mb.tile0 - 1) * xm::TILE; };
  {
    std::vector<int> idx, nw, se;
    for (int L = 2; L <= mb.la; ++L) {
      idx.push_back(mb.slot_of[L]);
      nw.push_back(slot(mo->lnwc[L - 1]));
      se.push_back(slot(mo->lsec[L - 1]));
    }
    const size_t n = idx.size();
    int *t = nullptr;
    CK(cudaMalloc(&t, std::max<size_t>(1, 3 * n) * sizeof(int)));
    cudaError_t e = cudaMemcpy(t, idx.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t + n, nw.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(t + 2 * n, se.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      xm::launch_put_int(c->stream, t, t + n, int(n), const_cast<int *>(D.nw));
      xm::launch_put_int(c->stream, t, t + 2 * n, int(n), const_cast<int *>(D.se));
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(t);
    CK(e);
  }
  // the serial lists: type-2 boundaries (with LNWC, LSEC) and flow-boundary edges
  std::vector<int4> &t2 = c->mom_t2[member], &bc = c->mom_bc[member];
  t2.clear();
  for (const int4 &e : mb.t2) {
    const int L = e.y;
    const int b = e.x == 1 ? slot(mo->lnwc[L - 1]) : e.x == 3 ? slot(mo->lsec[L - 1]) : 0;
    t2.push_back(int4{e.x, mb.slot_of[L], slot(e.z), b});
  }
  bc.clear();
  auto wslot = [&](int L) { return (L >= 2 && L <= mb.la) ? mb.slot_of[L] : -1; };
  for (int j = 0; j < mo->nbcs; ++j)
    bc.push_back(int4{wslot(mo->lbcs[j]), wslot(std::max(1, mo->lberc[j])),
                      wslot(std::max(1, mo->lbnrc[j])), 0});
  c->has_mom[member] = 1;
  c->mom_ld[member] = mo->ld;
  xm::MomScalars &q = c->mom_sc_h[member];
  q.kc = kc;
  q.tri = mo->stcuv ? 1 : 0;
  q.hdmf = mo->sdx ? 1 : 0;  // may diffuse; each call's ISHDMF decides
  // the lists move to the device with the next call
  if (c->mom_lists) {
    cudaFree(c->mom_lists);
    c->mom_lists = nullptr;
  }
  c->md.t2 = nullptr;
  return EFDC_XM_OK;
}

int32_t efdc_xm_explicit_batch(efdc_xm_ctx *c, const efdc_xm_explicit_params *prm,
                               efdc_xm_explicit_fields *f) {
  if (!c || !prm || !f) {
    set_error("efdc_xm_explicit_batch: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  const int M = c->M;
  // U, V, UHDY, VHDX NULL in every member: the previous call's, still on the device
  bool reuse = true;
  for (int m = 0; m < M; ++m) reuse &= !f[m].u && !f[m].v && !f[m].uhdy && !f[m].vhdx;
  if (reuse && !c->mom_inputs) {
    set_error("efdc_xm_explicit_batch: no U, V, UHDY, VHDX on the device yet");
    return EFDC_XM_BAD_ARGUMENT;
  }
  for (int m = 0; m < M; ++m) {
    const efdc_xm_explicit_fields &x = f[m];
    if (!c->mom_alloc || !c->has_mom[m] || (!reuse && (!x.u || !x.v || !x.uhdy || !x.vhdx)) ||
        (!x.fuhj != !x.fvhj)) {
      set_error("efdc_xm_explicit_batch: member %d: needs its static part "
                "(efdc_xm_set_momentum), U, V, UHDY, VHDX, and FUHJ with FVHJ or neither", m);
      return EFDC_XM_BAD_ARGUMENT;
    }
    if (prm[m].ishdmf >= 1 && (!c->mom_sc_h[m].hdmf || !x.fmdux || !x.fmduy || !x.fmdvx ||
                               !x.fmdvy)) {
      set_error("efdc_xm_explicit_batch: member %d has ISHDMF >= 1: needs SDX, SDY, LHDMF in "
                "its static part and FMDUX, FMDUY, FMDVX, FMDVY", m);
      return EFDC_XM_BAD_ARGUMENT;
    }
    if ((!x.hp) != (!f[0].hp) || (!x.wet) != (!f[0].wet) || (!x.fuhj) != (!f[0].fuhj)) {
      set_error("efdc_xm_explicit_batch: HP, WET and FUHJ are given for all members or none");
      return EFDC_XM_BAD_ARGUMENT;
    }
  }
  CK(cudaSetDevice(c->device));
  xm::MomDev &D = c->md;
  if (!D.t2) {  // the serial lists, packed per member
    std::vector<int4> t2, bc;
    std::vector<int> t2s(M + 1, 0), bcs(M + 1, 0);
    for (int m = 0; m < M; ++m) {
      t2s[m] = int(t2.size());
      bcs[m] = int(bc.size());
      t2.insert(t2.end(), c->mom_t2[m].begin(), c->mom_t2[m].end());
      bc.insert(bc.end(), c->mom_bc[m].begin(), c->mom_bc[m].end());
    }
    t2s[M] = int(t2.size());
    bcs[M] = int(bc.size());
    const size_t n4 = std::max<size_t>(1, t2.size()) + std::max<size_t>(1, bc.size());
    void *buf = nullptr;
    CK(cudaMalloc(&buf, n4 * sizeof(int4) + 2 * size_t(M + 1) * sizeof(int)));
    c->mom_lists = buf;
    int4 *t2d = static_cast<int4 *>(buf);
    int *sd = reinterpret_cast<int *>(t2d + n4);
    int4 *bcd = t2d + std::max<size_t>(1, t2.size());
    if (!t2.empty()) CK(cudaMemcpy(t2d, t2.data(), t2.size() * sizeof(int4), cudaMemcpyHostToDevice));
    if (!bc.empty()) CK(cudaMemcpy(bcd, bc.data(), bc.size() * sizeof(int4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(sd, t2s.data(), (M + 1) * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(sd + M + 1, bcs.data(), (M + 1) * sizeof(int), cudaMemcpyHostToDevice));
    D.t2 = t2d;
    D.bc = bcd;
    D.t2start = sd;
    D.bcstart = sd + M + 1;
  }
  // the call's inputs
  std::vector<Xfer> xs;
  int kcmax = 1;
  for (int m = 0; m < M; ++m) {
    xm::MomScalars &q = c->mom_sc_h[m];
    q.snlt = prm[m].snlt;
    q.on = 1;
    q.curv = prm[m].iscurvature != 0;
    q.fuhj = f[m].fuhj ? 1 : 0;
    q.hdmf = (prm[m].ishdmf >= 1 && c->mom_sc_h[m].hdmf) ? 1 : 0;
    kcmax = std::max(kcmax, q.kc);
  }
  auto per = [&](const double *efdc_xm_explicit_fields::*a) {
    std::vector<const double *> v(M);
    for (int m = 0; m < M; ++m) v[m] = f[m].*a;
    return v;
  };
  std::vector<Xfer> layers;
  if (!reuse) {
    layer_xfers(layers, per(&efdc_xm_explicit_fields::u), c->mom_ld, const_cast<double *>(D.u), D.ls, kcmax);
    layer_xfers(layers, per(&efdc_xm_explicit_fields::v), c->mom_ld, const_cast<double *>(D.v), D.ls, kcmax);
    layer_xfers(layers, per(&efdc_xm_explicit_fields::uhdy), c->mom_ld, const_cast<double *>(D.uhdy), D.ls, kcmax);
    layer_xfers(layers, per(&efdc_xm_explicit_fields::vhdx), c->mom_ld, const_cast<double *>(D.vhdx), D.ls, kcmax);
  }
  if (f[0].fuhj) {
    layer_xfers(layers, per(&efdc_xm_explicit_fields::fuhj), c->mom_ld, const_cast<double *>(D.fuhj), D.ls, kcmax);
    layer_xfers(layers, per(&efdc_xm_explicit_fields::fvhj), c->mom_ld, const_cast<double *>(D.fvhj), D.ls, kcmax);
  }
  bool any_hdmf = false;
  for (int m = 0; m < M; ++m) any_hdmf |= c->mom_sc_h[m].hdmf != 0;
  if (any_hdmf) {
    using In = const double *efdc_xm_explicit_fields::*;
    const In fm[4] = {
        &efdc_xm_explicit_fields::fmdux, &efdc_xm_explicit_fields::fmduy,
        &efdc_xm_explicit_fields::fmdvx, &efdc_xm_explicit_fields::fmdvy};
    const double *dv[4] = {D.fmdux, D.fmduy, D.fmdvx, D.fmdvy};
    for (int a = 0; a < 4; ++a) {
      std::vector<const double *> v = per(fm[a]);
      for (int m = 0; m < M; ++m)
        if (!c->mom_sc_h[m].hdmf) v[m] = nullptr;
      layer_xfers(layers, v, c->mom_ld, const_cast<double *>(dv[a]), D.ls, kcmax);
    }
  }
  // a member with fewer layers gives no array for the upper ones
  for (Xfer &x : layers) {
    bool any = false;
    for (const void *p : x.host) any |= p != nullptr;
    if (any) xs.push_back(x);
  }
  xm::MomDev Dc = D;  // this call's view
  if (f[0].hp) {
    std::vector<const void *> v(M);
    for (int m = 0; m < M; ++m) v[m] = f[m].hp;
    xs.push_back(Xfer{v, c->mom_hp, 0});
    Dc.hp = c->mom_hp;
  } else {
    Dc.hp = c->X.hp;  // the HP the last step left
  }
  if (f[0].wet) {
    std::vector<const void *> v(M);
    for (int m = 0; m < M; ++m) v[m] = f[m].wet;
    xs.push_back(Xfer{v, const_cast<int *>(D.wet), 1});
  } else {
    Dc.wet = nullptr;
  }
  // a member with fewer layers than another moves only its own: the per-member
  // transfers of a field must all be given, so the upper layers go member-wise
  int rc = 0;
  {
    std::vector<Xfer> full, partial;
    for (const Xfer &x : xs) {
      int n = 0;
      for (const void *p : x.host) n += p ? 1 : 0;
      (n == M ? full : partial).push_back(x);
    }
    for (size_t g0 = 0; !rc && g0 < full.size(); g0 += MAX_JOBS)
      rc = upload_arrays(c, std::vector<Xfer>(full.begin() + g0,
                                              full.begin() + std::min(full.size(), g0 + MAX_JOBS)));
    for (int m = 0; !rc && m < M; ++m) {
      std::vector<Xfer> mine;
      for (const Xfer &x : partial)
        if (x.host[m]) mine.push_back(x);
      if (!mine.empty()) rc = upload_member(c, m, mine);
    }
  }
  if (rc) return rc;
  c->mom_inputs = true;
  CK(cudaMemcpyAsync(const_cast<xm::MomScalars *>(D.sc), c->mom_sc_h.data(),
                     sizeof(xm::MomScalars) * M, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(D.cacsum, 0, sizeof(double) * M, c->stream));
  xm::launch_explicit(c->L(), c->S, Dc, c->X, kcmax, M);
  CK(cudaGetLastError());
  // the sums now differ from what the caller's arrays held
  c->synced &= ~uint32_t(EFDC_XM_SAME_FCAXE | EFDC_XM_SAME_FCAYE | EFDC_XM_SAME_FXE |
                         EFDC_XM_SAME_FYE);
  std::vector<Xfer> dn;
#define XM_DN(name, dev)                                                        \
  {                                                                             \
    std::vector<const void *> v(M);                                             \
    for (int m = 0; m < M; ++m) v[m] = f[m].name;                               \
    if ((rc = collect(c, dn, v, dev, 0, #name))) return rc;                     \
  }
  XM_DN(fcaxe, c->X.fcaxe) XM_DN(fcaye, c->X.fcaye) XM_DN(fxe, c->X.fxe) XM_DN(fye, c->X.fye)
#undef XM_DN
  auto per_out = [&](double *efdc_xm_explicit_fields::*a) {
    std::vector<const double *> v(M);
    for (int m = 0; m < M; ++m) v[m] = f[m].*a;
    return v;
  };
  std::vector<Xfer> ldn;
  using Out = double *efdc_xm_explicit_fields::*;
  const Out outs[5] = {
      &efdc_xm_explicit_fields::fcax, &efdc_xm_explicit_fields::fcay, &efdc_xm_explicit_fields::fx,
      &efdc_xm_explicit_fields::fy, &efdc_xm_explicit_fields::cac};
  double *devs[5] = {D.fcax, D.fcay, D.fx, D.fy, D.cac};
  for (int a = 0; a < 5; ++a) {
    std::vector<const double *> v = per_out(outs[a]);
    int n = 0;
    for (const double *p : v) n += p ? 1 : 0;
    if (n == 0) continue;
    if (n != M) {
      set_error("efdc_xm_explicit_batch: a layer output is given for some members only");
      return EFDC_XM_BAD_ARGUMENT;
    }
    for (int k = 0; k < kcmax; ++k) {  // members with fewer layers: below
      std::vector<const void *> hv(M);
      bool all = true;
      for (int m = 0; m < M; ++m) {
        hv[m] = k < c->mom_sc_h[m].kc ? static_cast<const void *>(v[m] + size_t(k) * c->mom_ld[m])
                                      : nullptr;
        all &= hv[m] != nullptr;
      }
      if (!all) {
        set_error("efdc_xm_explicit_batch: layer outputs need the same KC in every member");
        return EFDC_XM_BAD_ARGUMENT;
      }
      ldn.push_back(Xfer{hv, devs[a] + size_t(k) * D.ls, 0});
    }
  }
  dn.insert(dn.end(), ldn.begin(), ldn.end());
  for (size_t g0 = 0; !rc && g0 < dn.size(); g0 += MAX_JOBS)
    rc = download_arrays(c, std::vector<Xfer>(dn.begin() + g0,
                                              dn.begin() + std::min(dn.size(), g0 + MAX_JOBS)));
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  // the sums the caller received now equal the device's copies
  const uint32_t got = (f[0].fcaxe ? EFDC_XM_SAME_FCAXE : 0u) | (f[0].fcaye ? EFDC_XM_SAME_FCAYE : 0u) |
                       (f[0].fxe ? EFDC_XM_SAME_FXE : 0u) | (f[0].fye ? EFDC_XM_SAME_FYE : 0u);
  c->synced |= got;
  return EFDC_XM_OK;
}

int32_t efdc_xm_set_channels(efdc_xm_ctx *c, int32_t member, const efdc_xm_channels *ch) {
  if (!c || !ch || member < 0 || member >= (c ? c->M : 0) || ch->n < 0) {
    set_error("efdc_xm_set_channels: need a context, a member index and a channel struct");
    return EFDC_XM_BAD_ARGUMENT;
  }
  if (c->calib) {
    set_error("efdc_xm_set_channels: the adjoint does not cover sub-grid channels");
    return EFDC_XM_UNSUPPORTED;
  }
  const Member &mb = c->mem[member];
  std::vector<ChanSpec> list;
  if (ch->n > 0) {
    if (!ch->type || !ch->lhost || !ch->lu || !ch->lv || !ch->chanlen || !ch->chanfric ||
        !ch->dxp || !ch->dyp) {
      set_error("efdc_xm_set_channels: NULL channel array");
      return EFDC_XM_BAD_ARGUMENT;
    }
    auto water = [&](int L) {
      return L >= 2 && L <= mb.la && c->kind_h[mb.slot_of[L]] == xm::WATER;
    };
    for (int k = 0; k < ch->n; ++k) {
      ChanSpec s{ch->type[k], ch->lhost[k], ch->lu[k], ch->lv[k], ch->chanlen[k], ch->chanfric[k],
                 0.0, 0.0};
      const int lg = s.type == 1 ? s.lu : s.lv;
      if (s.type != 1 && s.type != 2) {
        set_error("efdc_xm_set_channels: channel %d: MDCHTYP %d (only 1 and 2 enter CALPUV2C)",
                  k + 1, s.type);
        return EFDC_XM_UNSUPPORTED;
      }
      if (!water(s.lh) || !water(lg) || s.lh == lg) {
        set_error("efdc_xm_set_channels: channel %d: host %d and guest %d must be distinct "
                  "water cells (2..LA) that are not open-boundary cells", k + 1, s.lh, lg);
        return EFDC_XM_BAD_ARGUMENT;
      }
      if (s.type == 2 && s.lu != 1 && !(s.lu >= 2 && s.lu <= mb.la)) {
        set_error("efdc_xm_set_channels: channel %d: LMDCHU %d (1 or a cell 2..LA)", k + 1, s.lu);
        return EFDC_XM_BAD_ARGUMENT;
      }
      // subchan.f90:51-52 (x) and :90-91 (y)
      s.gw = s.type == 1 ? ch->dxp[lg - 1] : ch->dyp[lg - 1];
      s.gl = s.type == 1 ? ch->dyp[lg - 1] : ch->dxp[lg - 1];
      list.push_back(s);
    }
  }
  CK(cudaSetDevice(c->device));
  c->chans[member] = std::move(list);
  return rebuild_channels(c);
}

int32_t efdc_xm_congrad(efdc_xm_ctx *c, const double *ccc, const double *ccs, const double *ccn,
                        const double *ccw, const double *cce, const double *ccci,
                        const double *fptmp, double *p, double rsqm, int32_t iterm,
                        int32_t precision, int32_t *iters, double *rsq) {
  int rc = single_only(c, "efdc_xm_congrad");
  if (rc) return rc;
  c->synced &= ~uint32_t(EFDC_XM_SAME_P);  // the solve runs in the state's P
  if (!ccc || !ccs || !ccn || !ccw || !cce || !fptmp || !p || iterm < 1) {
    set_error("efdc_xm_congrad: NULL argument or ITERM < 1");
    return EFDC_XM_BAD_ARGUMENT;
  }
  (void)ccci;  // CCCI = 1./CCC is recomputed on the device (same rounding)
  CK(cudaSetDevice(c->device));
  // the scaled system; land slots are reset to the inert CCC=1, C*=0, b=0
  auto one = [](const void *q) { return std::vector<const void *>{q}; };
  std::vector<Xfer> xs = {{one(ccc), c->Y.ccc, 3}, {one(ccs), c->Y.ccs, 3},
                          {one(ccn), c->Y.ccn, 3}, {one(ccw), c->Y.ccw, 3},
                          {one(cce), c->Y.cce, 3}, {one(fptmp), c->Y.fptmp, 3},
                          {one(p), c->X.p, 0}};
  if ((rc = upload_arrays(c, xs))) return rc;
  c->sc_h[0] = xm::StepScalars{};
  c->sc_h[0].rsqm = rsqm;
  c->sc_h[0].iterm = iterm;
  CK(cudaMemcpyAsync(c->sc, c->sc_h, sizeof(xm::StepScalars), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->ctl, 0, sizeof(Ctl), c->stream));
  c->act_h[0] = 1;
  if ((rc = write_act(c))) return rc;
  const bool mixed = precision == EFDC_XM_PREC_MIXED;
  c->mxview = xm::SysView{c->Y.fptmp, c->Y.ccc, c->Y.ccs, c->Y.ccw, c->Y.cce, c->Y.ccn, 0};
  c->last_mixed = false;
  c->sys_external = true;
  xm::launch_sys_prepare(c->L(), c->S, c->Y, c->ctl, mixed ? 1 : 0);
  CK(cudaGetLastError());
  rc = mixed ? solve_mixed(c, c->X.p, 0.0) : solve_fp64(c, c->X.p);
  if (rc) return rc;
  const Ctl k = c->ctl_h[0];
  std::vector<Xfer> out = {{one(p), c->X.p, 0}};
  if ((rc = download_arrays(c, out))) return rc;
  if (iters) *iters = k.iter;
  if (rsq) *rsq = mixed ? k.rsq64 : k.rsq;
  if (k.status != EFDC_XM_OK)
    set_error("CONGRAD: %s after %d iterations (RSQ=%g)",
              k.status == EFDC_XM_CG_MAXITER ? "maximum iterations exceeded" : "non-finite residual",
              k.iter, mixed ? k.rsq64 : k.rsq);
  return k.status;
}

void *efdc_xm_stream(efdc_xm_ctx *c) { return c ? static_cast<void *>(c->stream) : nullptr; }

int64_t efdc_xm_kernel_launches(void) { return g_launches.load(); }

int64_t efdc_xm_host_waits(void) { return g_waits.load(); }

int32_t efdc_xm_tune_key(const efdc_xm_ctx *c, int32_t precision, char *buf, int32_t len) {
  if (!c || !buf || len < 1) {
    set_error("efdc_xm_tune_key: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  snprintf(buf, size_t(len), "%s", tune_key(c, precision).c_str());
  return EFDC_XM_OK;
}

int32_t efdc_xm_tune_lookup(const char *table, const char *key, efdc_xm_schedule *out) {
  if (!table || !key || !out) {
    set_error("efdc_xm_tune_lookup: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  if (!table_lookup(table, key, out)) {
    set_error("efdc_xm_tune_lookup: no line for this key in %s", table);
    return EFDC_XM_BAD_ARGUMENT;
  }
  return EFDC_XM_OK;
}

int32_t efdc_xm_autotune(efdc_xm_ctx *c, int32_t precision, const char *table, int32_t flags,
                         efdc_xm_schedule *chosen, double *solve_ms) {
  if (!c || (precision != EFDC_XM_PREC_FP64 && precision != EFDC_XM_PREC_MIXED)) {
    set_error("efdc_xm_autotune: need a context and FP64 or MIXED");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  const std::string key = tune_key(c, precision);
  efdc_xm_schedule best{};
  if (solve_ms) *solve_ms = 0.0;
  if (!(flags & EFDC_XM_TUNE_MEASURE) && table && table_lookup(table, key, &best)) {
    apply_schedule(c, best);  // replayed: no measurement
    if (chosen) *chosen = best;
    return EFDC_XM_OK;
  }
  if (!c->stepped) {
    set_error("efdc_xm_autotune: step every member once first (the tuner times the solve of "
              "the system the last step assembled)");
    return EFDC_XM_BAD_ARGUMENT;
  }
  const bool mixed = precision == EFDC_XM_PREC_MIXED;
  if (mixed != c->last_mixed) {
    set_error("efdc_xm_autotune: the last step's precision differs from the one to tune");
    return EFDC_XM_BAD_ARGUMENT;
  }
  c->sys_external = false;
  c->mxview = xm::SysView{c->X.fp, c->X.cc, c->X.cs, c->X.cw, c->X.ce, c->X.cn, 1};
  if (!c->ptune && !(c->ptune = c->alloc<double>(size_t(c->nslot), false))) {
    set_error("efdc_xm_autotune: cudaMalloc failed");
    return EFDC_XM_CUDA_ERROR;
  }
  // P as the step left it is its system's solution: the timed solves start
  // from the step's own initial guess (ptmp), and P is put back at the end
  CK(cudaMemcpyAsync(c->ptune, c->X.p, size_t(c->nslot) * sizeof(double),
                     cudaMemcpyDeviceToDevice, c->stream));
  xm::launch_tune_guess(c->L(), c->S, c->X, c->ptmp);
  CK(cudaGetLastError());
  schedule_of(c, &best);
  double best_ms = 0.0;
  int rc = tune_time(c, mixed, 0.1, TUNE_REPS, &best_ms);
  if (rc) return rc;
  // coordinate descent: each knob's candidates in order, the others held
  auto knob = [&](int32_t efdc_xm_schedule::*f, std::initializer_list<int> vals) -> int {
    for (int v : vals) {
      efdc_xm_schedule s = best;
      s.*f = v;
      if (s.*f == best.*f) continue;
      apply_schedule(c, s);
      double ms = 0.0;
      const int r = tune_time(c, mixed, 0.1, TUNE_REPS, &ms);
      if (r) return r;
      // a candidate replaces the incumbent only if clearly faster (run-to-run
      // noise of a solve is about a percent)
      if (ms > 0 && (best_ms <= 0 || ms < TUNE_GAIN * best_ms)) {
        best = s;
        best_ms = ms;
      }
    }
    apply_schedule(c, best);
    return EFDC_XM_OK;
  };
  if (mixed) {
    if ((rc = knob(&efdc_xm_schedule::kernel_variant, {0, 1, 2, 3}))) return rc;
    if (best.kernel_variant > 0) {
      if ((rc = knob(&efdc_xm_schedule::ctas_matvec, {0, 2, 3, 4}))) return rc;
      if ((rc = knob(&efdc_xm_schedule::ctas_update, {0, 2, 3, 4}))) return rc;
    }
    if ((rc = knob(&efdc_xm_schedule::poly_threshold, {0, 10, 40, 100000}))) return rc;
    if ((rc = knob(&efdc_xm_schedule::inner_margin, {0, 1, 2}))) return rc;
    if ((rc = knob(&efdc_xm_schedule::inner_tol, {40, 50, 60, 70}))) return rc;
  }
  if ((rc = knob(&efdc_xm_schedule::graph_iters, {2, 4, 8}))) return rc;
  // P as the last step left it
  CK(cudaMemcpyAsync(c->X.p, c->ptune, size_t(c->nslot) * sizeof(double),
                     cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  apply_schedule(c, best);
  if (chosen) *chosen = best;
  if (solve_ms) *solve_ms = best_ms;
  if (table) {
    FILE *f = fopen(table, "a");
    if (!f) {
      set_error("efdc_xm_autotune: cannot append to %s", table);
      return EFDC_XM_BAD_ARGUMENT;
    }
    fprintf(f, "%s\n", table_line(key, best, best_ms).c_str());
    fclose(f);
  }
  return EFDC_XM_OK;
}

int32_t efdc_xm_set_option(efdc_xm_ctx *c, int32_t option, int32_t value) {
  if (!c) {
    set_error("efdc_xm_set_option: NULL context");
    return EFDC_XM_BAD_ARGUMENT;
  }
  switch (option) {
    case EFDC_XM_OPT_DEVICE_LOOPS:
      c->device_loops = value != 0;
      return EFDC_XM_OK;
    case EFDC_XM_OPT_GRAPH_ITERS:
      if (value < 1 || value > 32) break;
      if (value != c->graph_iters) {
        c->graph_iters = value;
        drop_step_graphs(c);
      }
      return EFDC_XM_OK;
    case EFDC_XM_OPT_POLY_THRESHOLD:
      if (value < 0 || value > 100000) break;
      c->poly_threshold = float(value);
      return EFDC_XM_OK;
    case EFDC_XM_OPT_INNER_MARGIN:
      if (value < 0 || value > 6) break;
      if (value != c->inner_margin_log10) {
        c->inner_margin_log10 = value;
        drop_graphs(c);
      }
      return EFDC_XM_OK;
    case EFDC_XM_OPT_SMALL_SOLVE:
      if (value < 0 || value > 1) break;
      if ((value != 0) != c->small_solve) {
        c->small_solve = value != 0;
        drop_graphs(c);
      }
      return EFDC_XM_OK;
    case EFDC_XM_OPT_CHUNKS:
      if (value < 1 || value > NCHUNK) break;
      c->nchunk = value;
      return EFDC_XM_OK;
    case EFDC_XM_OPT_FOLD_REDUCE:
      if (value < 0 || value > 2) break;
      if (value != c->fold_reduce) {
        c->fold_reduce = value;
        drop_graphs(c);
      }
      return EFDC_XM_OK;
    case EFDC_XM_OPT_INNER_TOL:
      if (value < 40 || value > 75) break;
      if (value != c->inner_tol_x10) {
        c->inner_tol_x10 = value;
        drop_graphs(c);
      }
      return EFDC_XM_OK;
    case EFDC_XM_OPT_KERNEL_VARIANT:
    case EFDC_XM_OPT_CTAS_MATVEC:
    case EFDC_XM_OPT_CTAS_UPDATE: {
      const bool var = option == EFDC_XM_OPT_KERNEL_VARIANT;
      if (var ? (value < 0 || value > 3) : (value < 0 || value > 32)) break;
      int &v = var ? c->kvariant : option == EFDC_XM_OPT_CTAS_MATVEC ? c->ctas_mv : c->ctas_up;
      if (v != value) {
        v = value;
        drop_graphs(c);  // the captured iterations hold the kernels and their grids
      }
      return EFDC_XM_OK;
    }
    default:
      break;
  }
  set_error("efdc_xm_set_option: unknown option %d or value %d out of range", option, value);
  return EFDC_XM_BAD_ARGUMENT;
}

void efdc_xm_transfer_bytes(int64_t *h2d, int64_t *d2h) {
  if (h2d) *h2d = g_h2d.load();
  if (d2h) *d2h = g_d2h.load();
}

int32_t efdc_xm_time_kernels(efdc_xm_ctx *c, int32_t precision, int32_t reps, efdc_xm_ktime *out) {
  if (!c || !out || reps < 1 || reps > 40) {
    set_error("efdc_xm_time_kernels: need a context, an output and 1 <= reps <= 40");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  const xm::Launch l = c->L();
  const bool mixed = precision == EFDC_XM_PREC_MIXED;
  if (!mixed && c->last_mixed) {
    const int rc0 = scaled_system(c);
    if (rc0) return rc0;
  }
  // the iterations run on a scratch copy of P with the stop tests disabled;
  // all launches are queued back to back (one untimed warm-up pair first),
  // so the events bracket device execution only, not host launch latency
  CK(cudaMemcpyAsync(c->ptmp, c->X.p, size_t(c->nslot) * sizeof(double), cudaMemcpyDeviceToDevice,
                     c->stream));
  for (int m = 0; m < c->M; ++m) c->act_h[m] = 1;
  int rc = write_act(c);
  if (rc) return rc;
  xm::launch_solve_reset(l, c->ctl, c->glob, c->act, c->M);
  if (mixed)
    xm::launch_mx_resid(l, c->S, c->mxview, c->Y, c->ptmp, c->ctl, c->glob, c->part, 1.0, 0.0,
                        1);
  else
    xm::launch_cg_init(l, c->S, c->Y, c->ptmp, c->ctl, c->glob, c->part);
  CK(cudaGetLastError());
  std::vector<cudaEvent_t> ev(2 * reps + 1);
  for (auto &e : ev) CK(cudaEventCreate(&e));
  auto pair = [&](int k) {
    if (mixed) {
      xm::launch_mx_matvec(l, c->S, c->Y, c->ctl, c->part);
      if (k >= 0) cudaEventRecord(ev[2 * k + 1], c->stream);
      xm::launch_mx_update(l, c->S, c->Y, c->ctl, c->glob, c->part, 1);
    } else {
      xm::launch_cg_matvec(l, c->S, c->Y, c->ptmp, c->ctl, c->part);
      if (k >= 0) cudaEventRecord(ev[2 * k + 1], c->stream);
      xm::launch_cg_update(l, c->S, c->Y, c->ctl, c->glob, c->part, 1);
    }
    if (k >= 0) cudaEventRecord(ev[2 * k + 2], c->stream);
  };
  pair(-1);
  CK(cudaEventRecord(ev[0], c->stream));
  for (int k = 0; k < reps; ++k) pair(k);
  CK(cudaGetLastError());
  CK(cudaEventSynchronize(ev[2 * reps]));
  double tm = 0, tu = 0;
  for (int k = 0; k < reps; ++k) {
    float a = 0, b = 0;
    CK(cudaEventElapsedTime(&a, ev[2 * k], ev[2 * k + 1]));
    CK(cudaEventElapsedTime(&b, ev[2 * k + 1], ev[2 * k + 2]));
    tm += a;
    tu += b;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  if ((rc = read_ctl(c))) return rc;
  out->ms_matvec = tm / reps;
  out->ms_update = tu / reps;
  out->reps = reps;
  long long ncell = 0;
  for (const Member &mb : c->mem) ncell += mb.la - 1;
  out->ncells = int32_t(std::min<long long>(ncell, INT32_MAX));
  out->nslots = (c->ntile - c->M) * TILE;  // the water tiles' slots
  long long npoly = 0;
  for (int m = 0; m < c->M; ++m)
    if (mixed && c->mpoly_h[m] && !(c->ctl_h[m].asym & 1)) npoly += c->mem[m].la - 1;
  out->ncells_poly = int32_t(std::min<long long>(npoly, INT32_MAX));
  for (int m = 0; m < c->M; ++m)
    if (c->ctl_h[m].done) {
      set_error("efdc_xm_time_kernels: the iteration of member %d stopped early (status %d)", m,
                c->ctl_h[m].status);
      return EFDC_XM_NONFINITE;
    }
  return EFDC_XM_OK;
}


// ---- calibration (adjoint) entry points: single-basin contexts ----

static int calib_ready(efdc_xm_ctx *c, const char *who) {
  if (!c) {
    set_error("%s: NULL context", who);
    return EFDC_XM_BAD_ARGUMENT;
  }
  if (!c->calib) {
    set_error("%s: call efdc_xm_calib_enable first", who);
    return EFDC_XM_BAD_ARGUMENT;
  }
  return EFDC_XM_OK;
}

static int gauge_slots(efdc_xm_ctx *c, int32_t n, const int32_t *L) {
  if (n < 0 || (n > 0 && !L)) {
    set_error("gauge list: bad arguments");
    return EFDC_XM_BAD_ARGUMENT;
  }
  if (n > c->gcap) {
    if (c->gslot) cudaFree(c->gslot);
    if (c->gbuf) cudaFree(c->gbuf);
    c->gslot = nullptr;
    c->gbuf = nullptr;
    c->gcap = 0;
    CK(cudaMalloc(&c->gslot, size_t(n) * sizeof(int)));
    CK(cudaMalloc(&c->gbuf, size_t(n) * sizeof(double)));
    c->gcap = n;
  }
  std::vector<int> sl(n);
  const Member &mb = c->mem[0];
  for (int i = 0; i < n; ++i) {
    if (L[i] < 2 || L[i] > mb.la) {
      set_error("gauge list: L=%d outside 2..LA", L[i]);
      return EFDC_XM_BAD_ARGUMENT;
    }
    sl[i] = mb.slot_of[L[i]];
  }
  if (n > 0)
    CK(cudaMemcpyAsync(c->gslot, sl.data(), size_t(n) * sizeof(int), cudaMemcpyHostToDevice,
                       c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EFDC_XM_OK;
}

int32_t efdc_xm_calib_enable(efdc_xm_ctx *c, int32_t nsnap) {
  int rc = single_only(c, "efdc_xm_calib_enable");
  if (rc) return rc;
  if (nsnap < 1) {
    set_error("efdc_xm_calib_enable: need at least one snapshot slot");
    return EFDC_XM_BAD_ARGUMENT;
  }
  if (c->any_may_asym) {
    set_error("efdc_xm_calib_enable: the adjoint covers clamped open boundaries (ISPB=0) only");
    return EFDC_XM_UNSUPPORTED;
  }
  if (c->S.ch.n > 0) {
    set_error("efdc_xm_calib_enable: the adjoint does not cover sub-grid channels");
    return EFDC_XM_UNSUPPORTED;
  }
  if (c->calib) {
    set_error("efdc_xm_calib_enable: already enabled");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  const size_t ns = c->nslot;
  xm::DevCalib &A = c->A;
  double **arrs[] = {&A.kappa, &A.ap_in, &A.ahp_in, &A.ahu_in, &A.ahv_in, &A.au_in, &A.av_in,
                     &A.ap_out, &A.ahp_out, &A.ahu_out, &A.ahv_out, &A.au_out, &A.av_out,
                     &A.ahpe, &A.rhs, &A.lam, &A.afp, &A.afu, &A.afv, &A.atbx, &A.atby,
                     &A.nbu, &A.nbv, &A.vub, &A.uvb, &A.akappa, &A.abelv};
  for (double **a : arrs)
    if (!(*a = c->alloc<double>(ns))) {
      set_error("efdc_xm_calib_enable: cudaMalloc failed");
      return EFDC_XM_CUDA_ERROR;
    }
  const size_t nb = size_t(std::max(1, c->nobc)) * std::max(1, c->B.mtmax);
  A.apcb = c->alloc<double>(nb);
  A.apsb = c->alloc<double>(nb);
  A.nflag = c->alloc<int>(1);
  c->psol = c->alloc<double>(ns);
  c->bsq = c->alloc<double>(1);
  if (!A.apcb || !A.apsb || !A.nflag || !c->psol || !c->bsq) {
    set_error("efdc_xm_calib_enable: cudaMalloc failed");
    return EFDC_XM_CUDA_ERROR;
  }
  for (int k = 0; k < nsnap; ++k) {
    std::array<double *, 6> a{};
    for (double *&x : a)
      if (!(x = c->alloc<double>(ns))) {
        set_error("efdc_xm_calib_enable: cudaMalloc failed (snapshots)");
        return EFDC_XM_CUDA_ERROR;
      }
    c->snap.push_back(a);
  }
  A.tbx = const_cast<double *>(c->X.tbx);
  A.tby = const_cast<double *>(c->X.tby);
  CK(cudaDeviceSynchronize());  // the zero-fills of the legacy stream
  c->calib = true;
  return EFDC_XM_OK;
}

int32_t efdc_xm_calib_set_roughness(efdc_xm_ctx *c, const double *log_n) {
  int rc = calib_ready(c, "efdc_xm_calib_set_roughness");
  if (rc) return rc;
  if (!log_n) {
    set_error("efdc_xm_calib_set_roughness: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  std::vector<Xfer> xs = {{{log_n}, c->A.kappa, 0}};
  return upload_arrays(c, xs);
}

int32_t efdc_xm_calib_set_harmonics(efdc_xm_ctx *c, const double *pcb, const double *psb) {
  int rc = calib_ready(c, "efdc_xm_calib_set_harmonics");
  if (rc) return rc;
  if (c->nobc == 0) return EFDC_XM_OK;
  if (!pcb || !psb) {
    set_error("efdc_xm_calib_set_harmonics: NULL argument");
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  const size_t n = size_t(c->nobc) * c->B.mtmax * sizeof(double);
  CK(cudaMemcpyAsync(const_cast<double *>(c->B.pcb), pcb, n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(const_cast<double *>(c->B.psb), psb, n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EFDC_XM_OK;
}

static int snap_copy(efdc_xm_ctx *c, int32_t slot, bool save) {
  if (slot < 0 || slot >= int(c->snap.size())) {
    set_error("snapshot slot %d outside 0..%d", slot, int(c->snap.size()) - 1);
    return EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  double *live[6] = {c->X.p, c->X.hp, c->X.hu, c->X.hv, c->X.uhdye, c->X.vhdxe};
  const size_t nb = size_t(c->nslot) * sizeof(double);
  for (int k = 0; k < 6; ++k)
    CK(cudaMemcpyAsync(save ? c->snap[slot][k] : live[k], save ? live[k] : c->snap[slot][k], nb,
                       cudaMemcpyDeviceToDevice, c->stream));
  return EFDC_XM_OK;
}

int32_t efdc_xm_calib_snapshot(efdc_xm_ctx *c, int32_t slot) {
  const int rc = calib_ready(c, "efdc_xm_calib_snapshot");
  return rc ? rc : snap_copy(c, slot, true);
}

int32_t efdc_xm_calib_restore(efdc_xm_ctx *c, int32_t slot) {
  const int rc = calib_ready(c, "efdc_xm_calib_restore");
  if (rc) return rc;
  c->synced &= ~STEP_WRITES;  // the snapshot overwrites the state
  return snap_copy(c, slot, false);
}

int32_t efdc_xm_calib_step(efdc_xm_ctx *c, const efdc_xm_params *prm, efdc_xm_stats *stats) {
  if (c) c->synced &= ~uint32_t(EFDC_XM_SAME_TBX | EFDC_XM_SAME_TBY);  // the drag is written
  efdc_xm_stats dummy;
  if (!stats) stats = &dummy;
  std::memset(stats, 0, sizeof(*stats));
  int rc = calib_ready(c, "efdc_xm_calib_step");
  if (rc) return stats->status = rc;
  if (!prm || prm->isdry != 0 || prm->precision != EFDC_XM_PREC_FP64 || prm->bsc > 1.E-6) {
    set_error("efdc_xm_calib_step: the calibration model runs FP64 with ISDRY=0 and BSC=0");
    return stats->status = EFDC_XM_BAD_ARGUMENT;
  }
  CK(cudaSetDevice(c->device));
  // the drag of this step from the state at its start (the scalars first)
  c->sc_h[0] = make_scalars(c->mem[0], prm);
  CK(cudaMemcpyAsync(c->sc, c->sc_h, sizeof(xm::StepScalars), cudaMemcpyHostToDevice, c->stream));
  xm::DevCalib A = c->A;
  A.u0 = c->X.uhdye;
  A.v0 = c->X.vhdxe;
  A.hu0 = c->X.hu;
  A.hv0 = c->X.hv;
  xm::launch_cal_tbxy(c->L(), c->S, c->X, A);
  CK(cudaGetLastError());
  return efdc_xm_step_device_batch(c, prm, stats);
}

int32_t efdc_xm_calib_gauges(efdc_xm_ctx *c, int32_t n, const int32_t *L, double *p_out) {
  int rc = calib_ready(c, "efdc_xm_calib_gauges");
  if (rc) return rc;
  if (n == 0) return EFDC_XM_OK;
  if (!p_out) {
    set_error("efdc_xm_calib_gauges: NULL output");
    return EFDC_XM_BAD_ARGUMENT;
  }
  if ((rc = gauge_slots(c, n, L))) return rc;
  xm::launch_gather_slots(c->stream, c->X.p, c->gslot, n, c->gbuf);
  CK(cudaMemcpyAsync(p_out, c->gbuf, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EFDC_XM_OK;
}

int32_t efdc_xm_calib_adjoint_reset(efdc_xm_ctx *c) {
  int rc = calib_ready(c, "efdc_xm_calib_adjoint_reset");
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  xm::DevCalib &A = c->A;
  const size_t nb = size_t(c->nslot) * sizeof(double);
  double *z[] = {A.ap_in, A.ahp_in, A.ahu_in, A.ahv_in, A.au_in, A.av_in, A.ap_out, A.ahp_out,
                 A.ahu_out, A.ahv_out, A.au_out, A.av_out, A.akappa, A.abelv};
  for (double *a : z) CK(cudaMemsetAsync(a, 0, nb, c->stream));
  const size_t np = size_t(std::max(1, c->nobc)) * std::max(1, c->B.mtmax) * sizeof(double);
  CK(cudaMemsetAsync(A.apcb, 0, np, c->stream));
  CK(cudaMemsetAsync(A.apsb, 0, np, c->stream));
  CK(cudaMemsetAsync(A.nflag, 0, sizeof(int), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return EFDC_XM_OK;
}

int32_t efdc_xm_calib_add_p_adjoint(efdc_xm_ctx *c, int32_t n, const int32_t *L, const double *w) {
  int rc = calib_ready(c, "efdc_xm_calib_add_p_adjoint");
  if (rc) return rc;
  if (n == 0) return EFDC_XM_OK;
  if (!w) {
    set_error("efdc_xm_calib_add_p_adjoint: NULL weights");
    return EFDC_XM_BAD_ARGUMENT;
  }
  if ((rc = gauge_slots(c, n, L))) return rc;
  CK(cudaMemcpyAsync(c->gbuf, w, size_t(n) * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  xm::launch_adj_gauge(c->L(), c->gslot, c->gbuf, n, c->A.ap_in);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return EFDC_XM_OK;
}

int32_t efdc_xm_calib_adjoint_step(efdc_xm_ctx *c, const efdc_xm_params *prm, int32_t slot,
                                   double rel_tol, int32_t *cg_iters) {
  int rc = calib_ready(c, "efdc_xm_calib_adjoint_step");
  if (rc) return rc;
  if (!(rel_tol > 0.0)) {
    set_error("efdc_xm_calib_adjoint_step: rel_tol must be > 0");
    return EFDC_XM_BAD_ARGUMENT;
  }
  // the step again, from its start state: its operator, CG solution and drag
  if ((rc = efdc_xm_calib_restore(c, slot))) return rc;
  efdc_xm_stats st;
  rc = efdc_xm_calib_step(c, prm, &st);
  if (rc != EFDC_XM_OK) return rc;
  const xm::Launch l = c->L();
  xm::DevCalib &A = c->A;
  A.p0 = c->snap[slot][0];
  A.hp0 = c->snap[slot][1];
  A.hu0 = c->snap[slot][2];
  A.hv0 = c->snap[slot][3];
  A.u0 = c->snap[slot][4];
  A.v0 = c->snap[slot][5];
  A.psol = c->psol;
  xm::launch_adj_pre(l, c->S, c->X, c->B, A);
  CK(cudaMemsetAsync(c->bsq, 0, sizeof(double), c->stream));
  xm::launch_adj_rhs(l, c->S, c->Y, c->ctl, A, c->bsq);
  CK(cudaGetLastError());
  double bsq = 0.0;
  CK(cudaMemcpyAsync(&bsq, c->bsq, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int iters = 0;
  if (bsq > 0.0) {  // A lam = rhs, the step's operator (symmetric), relative stop
    c->sc_h[0].rsqm = rel_tol * rel_tol * bsq;
    CK(cudaMemcpyAsync(c->sc, c->sc_h, sizeof(xm::StepScalars), cudaMemcpyHostToDevice,
                       c->stream));
    c->act_h[0] = 1;
    if ((rc = write_act(c))) return rc;
    if ((rc = solve_fp64(c, A.lam))) return rc;
    const Ctl &k = c->ctl_h[0];
    iters = k.iter;
    if (k.status != EFDC_XM_OK) {
      set_error("adjoint CONGRAD: %s after %d iterations",
                k.status == EFDC_XM_CG_MAXITER ? "maximum iterations exceeded"
                                               : "non-finite residual", k.iter);
      return k.status;
    }
  }
  if (cg_iters) *cg_iters = iters;
  xm::launch_adj_post(l, c->S, c->X, c->B, A);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  // the adjoints of this step's inputs are those of the previous step's outputs
  std::swap(A.ap_in, A.ap_out);
  std::swap(A.ahp_in, A.ahp_out);
  std::swap(A.ahu_in, A.ahu_out);
  std::swap(A.ahv_in, A.ahv_out);
  std::swap(A.au_in, A.au_out);
  std::swap(A.av_in, A.av_out);
  return EFDC_XM_OK;
}

int32_t efdc_xm_calib_gradients(efdc_xm_ctx *c, double *dlog_n, double *dbelv, double *dpcb,
                                double *dpsb, double *const state[6], int32_t *n_clamped) {
  int rc = calib_ready(c, "efdc_xm_calib_gradients");
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  const xm::DevCalib &A = c->A;
  auto one = [](const void *q) { return std::vector<const void *>{q}; };
  std::vector<Xfer> xs;
  if (dlog_n) xs.push_back({one(dlog_n), A.akappa, 0});
  if (dbelv) xs.push_back({one(dbelv), A.abelv, 0});
  if (state) {
    double *src[6] = {A.ap_in, A.ahp_in, A.ahu_in, A.ahv_in, A.au_in, A.av_in};
    for (int k = 0; k < 6; ++k)
      if (state[k]) xs.push_back({one(state[k]), src[k], 0});
  }
  if ((rc = download_arrays(c, xs))) return rc;
  CK(cudaStreamSynchronize(c->stream));  // the copies below run on the legacy stream
  const size_t np = size_t(c->nobc) * c->B.mtmax * sizeof(double);
  if (np && dpcb) CK(cudaMemcpy(dpcb, A.apcb, np, cudaMemcpyDeviceToHost));
  if (np && dpsb) CK(cudaMemcpy(dpsb, A.apsb, np, cudaMemcpyDeviceToHost));
  if (n_clamped) CK(cudaMemcpy(n_clamped, A.nflag, sizeof(int), cudaMemcpyDeviceToHost));
  return EFDC_XM_OK;
}

}  // extern "C"
