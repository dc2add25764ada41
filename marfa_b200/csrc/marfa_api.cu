// marfa_api.cu -- host side of libmarfa_gpu.so: the C ABI of include/marfa_gpu.h.
//
// The host work per call is the part of the reference's driver that is cheap
// and sequential: the subinterval loop bounds (main.f90:117-122, 171-172), the
// starting line (main.f90:196-248) and the per-subinterval line window
// recurrence of lblScheme (LBL.f90:41-61 with capWV of main.f90:138-144).
// Everything per line and per grid point runs on the device.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "marfa_gpu.h"
#include "marfa_kernels.cuh"
#include "marfa_windows.h"

using namespace marfa;

namespace {


struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
};

} // namespace

// Launch parameters that do not change results (chosen by marfa_autotune).
struct Tune {
  int far_chunk = 16384;   // lines per far-kernel block
  int coop_k = 5;          // fine grids whose cell pairs are summed by lane groups
  int small_block_lines = 512; // batches whose units all have fewer near lines use small blocks
  int fine_pair = 0;       // FP32c dense units on two 512-thread fine blocks per SM (else one of 1024)
};

// Bucket index over the sorted line centres: first[b] = first line with
// nu >= lo + b w (w = 1 / inv_w, about four lines per bucket), b = 0 .. nb + 1.
// A search for x only looks between the entries of x's bucket and its
// neighbours, which hold every lower and upper bound of x whatever the
// rounding of the bucket position.
struct NuIndex {
  double lo = 0.0, inv_w = 0.0;
  std::vector<int64_t> first;
  void build(const std::vector<double> &nu) {
    const int64_t n = (int64_t)nu.size();
    first.clear();
    inv_w = 0.0;
    if (n < 2 || !(nu.back() > nu.front())) return;
    lo = nu.front();
    const int64_t nb = std::min<int64_t>(std::max<int64_t>(n / 4, 1), (int64_t)1 << 22);
    inv_w = (double)nb / (nu.back() - lo);
    first.resize(nb + 2);
    int64_t q = 0;
    for (int64_t b = 0; b <= nb + 1; ++b) {
      const double edge = lo + (double)b / inv_w;
      while (q < n && nu[q] < edge) ++q;
      first[b] = q;
    }
  }
  // lines [a, b) hold the first nu >= x and the first nu > x (or b = n)
  void range(double x, int64_t n, int64_t &a, int64_t &b) const {
    if (inv_w == 0.0) {
      a = 0;
      b = n;
      return;
    }
    const int64_t nb = (int64_t)first.size() - 2;
    const double t = (x - lo) * inv_w;
    const int64_t k = t < 0.0 ? 0 : (t >= (double)nb ? nb : (int64_t)t);
    a = first[k > 0 ? k - 1 : 0];
    b = k + 2 <= nb + 1 ? first[k + 2] : n;
  }
};

struct marfa_ctx {
  int device = 0;
  Tune tune;
  unsigned long long alloc_gen = 0; // counts (re)allocations of the work buffers
  cudaStream_t stream = nullptr;
  // records to host memory: copies of one chunk of levels overlap the
  // computation of the next (two device halves, copy stream, events)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t rec_ready[2] = {nullptr, nullptr}, rec_copied[2] = {nullptr, nullptr};
  // per level of the last call with host records: kernel time and copy time
  // (ms), which shape the level chunks of the next such call
  double rec_compute_ms = 0.0, rec_copy_ms = 0.0;
  int sm_count = 0;
  // second stream and buffer set: with host records, consecutive chunks run
  // on alternating streams with their own line and scratch buffers, so that
  // one chunk's first kernels fill the SMs the previous chunk's last
  // kernels leave idle
  cudaStream_t stream2 = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  int64_t n_lines = 0;
  std::vector<double> nu;  // host copy of the sorted centres (window scan)
  NuIndex nu_index;        // bucket index over nu (near-line bounds)
  double smax = 0.0;       // largest reference intensity
  double dmin = 0.0, dmax = 0.0;
  int n_iso = 0, n_temp = 0;
  TipsGrid tgrid{20.0, 2.0}; // the reference's TIPS grid unless set otherwise
  // line list, structure of arrays
  double *d_nu = nullptr;
  float *d_S = nullptr, *d_gair = nullptr, *d_gself = nullptr, *d_elow = nullptr,
        *d_nair = nullptr, *d_delta = nullptr;
  int *d_iso = nullptr;
  double *d_S64 = nullptr, *d_gair64 = nullptr; // marfa_ctx_set_line_params overrides
  double *d_tips = nullptr;
  int *d_err = nullptr;
  // grow-only work buffers
  DevBuf b_nus, b_gen, b_hot, b_rank, b_snu, b_sidx, b_far, b_fold, b_scr, b_lv, b_margin, b_win, b_chunks,
      b_out, b_out64, b_dump, b_count, b_gstage, b_aux, b_gscr, b_cot, b_grad, b_vbuf, b_queue, b_order, b_tune;
  DevBuf b2_nus, b2_gen, b2_hot, b2_rank, b2_snu, b2_sidx, b2_far, b2_fold, b2_scr, b2_gstage, b2_vbuf, b2_queue;
  std::string err;
  // pinned staging of the per-call host tables (see Staging): a ring of
  // buffers, used by consecutive calls in turn
  static constexpr int NPIN = 4;
  void *pinned[NPIN] = {};
  size_t pinned_cap[NPIN] = {};
  cudaEvent_t pinned_ev[NPIN] = {};
  bool pinned_pending[NPIN] = {};
  int pinned_next = 0;
  std::vector<cudaEvent_t> events;
  // timing marks of the last compute call: (family, start, stop); family 5
  // is the whole call
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
  int launches = 0, far_launches = 0;
};

namespace {

int set_err(marfa_ctx *c, int code, const char *fmt, ...) {
  if (c) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    c->err = buf;
  }
  return code;
}

int cuda_fail(marfa_ctx *c, cudaError_t e, const char *where) {
  if (e == cudaErrorMemoryAllocation)
    return set_err(c, MARFA_E_NOMEM, "%s: %s", where, cudaGetErrorString(e));
  return set_err(c, MARFA_E_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

#define CK(call, where)                                      \
  do {                                                       \
    cudaError_t e__ = (call);                                \
    if (e__ != cudaSuccess) return cuda_fail(ctx, e__, where); \
  } while (0)

cudaError_t ensure(DevBuf &b, size_t bytes) {
  if (bytes <= b.cap) return cudaSuccess;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  const size_t want = std::max(bytes, (size_t)256);
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e == cudaSuccess) b.cap = want;
  return e;
}

// Grow-only buffer of the context; a reallocation invalidates captured graphs.
cudaError_t ensure(marfa_ctx *ctx, DevBuf &b, size_t bytes) {
  if (bytes <= b.cap) return cudaSuccess;
  ++ctx->alloc_gen;
  return ensure(b, bytes);
}

void release(DevBuf &b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

} // namespace

namespace {

// The host tables of one call (windows, chunks, levels, work order) reach the
// device through a pinned buffer of the context: a copy from pageable memory
// would first wait for the stream to drain, so that the host planning of a
// call could not overlap the kernels of the previous one.  Consecutive calls
// take the buffers of a ring in turn, and a buffer is rewritten only after
// its previous copies have completed, so that the host can queue calls up to
// the ring's length ahead of the device (and a late host thread does not
// leave the device idle).
struct Staging {
  marfa_ctx *ctx;
  cudaStream_t st;
  size_t off = 0;
  int slot = 0;
  cudaError_t begin(size_t bytes) {
    cudaError_t e = cudaSuccess;
    slot = ctx->pinned_next;
    ctx->pinned_next = (slot + 1) % marfa_ctx::NPIN;
    if (ctx->pinned_pending[slot]) {
      if ((e = cudaEventSynchronize(ctx->pinned_ev[slot]))) return e;
      ctx->pinned_pending[slot] = false;
    }
    if (!ctx->pinned_ev[slot] &&
        (e = cudaEventCreateWithFlags(&ctx->pinned_ev[slot], cudaEventDisableTiming)))
      return e;
    if (bytes > ctx->pinned_cap[slot]) {
      // pinned allocation synchronizes the device: grow every slot of the
      // ring at once (with headroom), so that later calls never allocate
      const size_t cap = bytes + bytes / 2 + 4096;
      for (int s = 0; s < marfa_ctx::NPIN; ++s) {
        if (ctx->pinned_pending[s]) {
          if ((e = cudaEventSynchronize(ctx->pinned_ev[s]))) return e;
          ctx->pinned_pending[s] = false;
        }
        if (ctx->pinned_cap[s] >= cap) continue;
        if (ctx->pinned[s]) cudaFreeHost(ctx->pinned[s]);
        ctx->pinned[s] = nullptr;
        ctx->pinned_cap[s] = 0;
        if ((e = cudaMallocHost(&ctx->pinned[s], cap))) return e;
        ctx->pinned_cap[s] = cap;
      }
    }
    off = 0;
    return e;
  }
  cudaError_t put(void *dst, const void *src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    char *h = (char *)ctx->pinned[slot] + off;
    std::memcpy(h, src, bytes);
    off += (bytes + 15) & ~(size_t)15;
    return cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, st);
  }
  cudaError_t end() {
    cudaError_t e = cudaEventRecord(ctx->pinned_ev[slot], st);
    if (e == cudaSuccess) ctx->pinned_pending[slot] = true;
    return e;
  }
  static size_t room(size_t bytes) { return (bytes + 15) & ~(size_t)15; }
};

// Constants of Constants.f90 evaluated in double.
Consts make_consts() {
  Consts c;
  c.pi = 3.1415926;
  c.sqln2 = std::sqrt(std::log(2.0));
  c.c2 = 6.626070e-27 * 2.99792458e10 / 1.3806503e-16;
  c.doppler = std::sqrt(2.0 * 6.02214076e23 * 1.3806503e-16 * std::log(2.0)) / 2.99792458e10;
  c.tref = 296.0;
  c.bolsi = 1.3806503e-23;
  c.stdp = 101325.0;
  c.sqrtpi = std::sqrt(c.pi);
  c.sqrt14 = std::sqrt(1.4);
  return c;
}

// Subinterval bounds, windows and far-kernel chunks of one run.
struct Plan {
  int n_sub = 0;
  std::vector<double> s, e;       // start / end of each subinterval
  std::vector<int64_t> lo, hi;    // line window [lo, hi), 0-based
  std::vector<int> chunk_sub;
  std::vector<int64_t> chunk_begin, chunk_end;
  std::vector<int> sub_chunk0;    // n_sub + 1
  int max_chunks = 0;             // most chunks of one subinterval
};

// Windows of all subintervals (marfa_windows.h).
int plan_windows(const double *nu, int64_t n, double start_wv, double end_wv, double cut,
                 std::vector<double> &ss, std::vector<double> &se, std::vector<int64_t> &lo,
                 std::vector<int64_t> &hi, int &bad) {
  return plan_windows_of(nu, n, start_wv, marfa_num_subintervals(start_wv, end_wv), cut, ss, se, lo, hi, bad);
}

int make_plan(marfa_ctx *ctx, const marfa_run *run, Plan &pl) {
  pl.n_sub = marfa_num_subintervals(run->start_wv, run->end_wv);
  int bad = -1;
  if (plan_windows(ctx->nu.data(), ctx->n_lines, run->start_wv, run->end_wv, run->cutoff, pl.s, pl.e,
                   pl.lo, pl.hi, bad))
    return set_err(ctx, MARFA_E_DB,
                   bad < 0 ? "line list ends before start - cutoff"
                           : "line list ends inside a subinterval window (add a sentinel line beyond "
                             "end + 10 + cutoff)");
  pl.sub_chunk0.assign(pl.n_sub + 1, 0);
  for (int isub = 0; isub < pl.n_sub; ++isub) {
    pl.sub_chunk0[isub] = (int)pl.chunk_sub.size();
    const int64_t chunk = ctx->tune.far_chunk;
    for (int64_t b = pl.lo[isub]; b < pl.hi[isub]; b += chunk) {
      pl.chunk_sub.push_back(isub);
      pl.chunk_begin.push_back(b);
      pl.chunk_end.push_back(std::min(b + chunk, pl.hi[isub]));
    }
  }
  pl.sub_chunk0[pl.n_sub] = (int)pl.chunk_sub.size();
  for (int isub = 0; isub < pl.n_sub; ++isub)
    pl.max_chunks = std::max(pl.max_chunks, pl.sub_chunk0[isub + 1] - pl.sub_chunk0[isub]);
  return MARFA_OK;
}

int check_run(marfa_ctx *ctx, const marfa_run *run) {
  if (!ctx) return MARFA_E_ARG;
  if (!run) return set_err(ctx, MARFA_E_ARG, "run is null");
  if (!(run->cutoff > 0.0) || !std::isfinite(run->cutoff) || run->cutoff > 4000.0)
    return set_err(ctx, MARFA_E_ARG, "cutoff must be in (0, 4000] cm-1");
  if (!std::isfinite(run->start_wv) || !std::isfinite(run->end_wv))
    return set_err(ctx, MARFA_E_ARG, "non-finite spectral interval");
  if (run->target != MARFA_TARGET_ACS && run->target != MARFA_TARGET_VAC)
    return set_err(ctx, 2, "target must be ACS or VAC");
  if (run->chi < MARFA_CHI_NONE || run->chi > MARFA_CHI_PERRIN)
    return set_err(ctx, MARFA_E_ARG, "unknown chi-factor %d", run->chi);
  if (run->shape != MARFA_SHAPE_VOIGT && run->shape != MARFA_SHAPE_LORENTZ && run->shape != MARFA_SHAPE_ONE &&
      run->shape != MARFA_SHAPE_ABSX)
    return set_err(ctx, MARFA_E_ARG, "unknown shape %d", run->shape);
  if (run->precision != MARFA_PREC_FP64 && run->precision != MARFA_PREC_FP32C)
    return set_err(ctx, MARFA_E_ARG, "unknown precision %d", run->precision);
  if (run->mol_code < 1 || run->mol_code > 12) return set_err(ctx, 8, "unsupported molecule code %d", run->mol_code);
  return MARFA_OK;
}

int build_levels(marfa_ctx *ctx, int n, const double *P, const double *T, const double *dens,
                 std::vector<LevelConst> &lv) {
  const Consts c = make_consts();
  lv.resize(n);
  for (int l = 0; l < n; ++l) {
    if (!std::isfinite(P[l]) || !std::isfinite(T[l]) || !std::isfinite(dens[l]) || P[l] < 0.0)
      return set_err(ctx, 7, "level %d: invalid pressure/temperature/density", l + 1);
    int idx = 1;
    double uw = 0.0;
    if (!tips_node(T[l], ctx->tgrid, ctx->n_temp, idx, uw))
      return set_err(ctx, MARFA_E_TEMPERATURE, "level %d: temperature %.3f K outside the TIPS table",
                     l + 1, T[l]);
    LevelConst &v = lv[l];
    v.P = P[l];
    v.T = T[l];
    v.density = dens[l];
    v.pself = dens[l] * 10.0 * c.bolsi * T[l] / c.stdp; // main.f90:92
    if (v.pself > P[l] * (1.0 + 1e-6))
      return set_err(ctx, 7, "level %d: partial pressure %.6g atm from the density exceeds the total "
                             "pressure %.6g atm", l + 1, v.pself, P[l]);
    v.perrin_b1 = 0.0888 - 0.16 * std::exp(-(0.00410 * T[l]));
    v.perrin_b2 = 0.0526 * std::exp(-(0.00152 * T[l]));
  }
  return MARFA_OK;
}

// Device buffers of a vector-Jacobian product (marfa_vjp).
struct VjpOut {
  const double *cot = nullptr;   // [levels][n_sub][NT] cotangent of the records
  double *dS = nullptr, *dgair = nullptr, *dT = nullptr, *dP = nullptr;
};

// Fine-kernel launch plan of one chunk of levels.
struct FineChunk {
  int max_near = 0, smem_cap = 0, gstage_cap = 0, block_threads = 0, resident = 0;
  size_t smem_room = 0;
  size_t gstage_bytes = 0;
};

// Capture of one compute call into a CUDA graph, and its replays.
struct GraphCtl {
  bool replay = false;             // false: capture during this call
  int Lc = 0, UB = 0;              // chunking of the captured call
  std::vector<long long> sig;      // launch plan of the captured call
  unsigned long long alloc_gen = 0;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
};

struct Outputs {
  GraphCtl *graph = nullptr;     // capture into / replay of a CUDA graph
  const VjpOut *vjp = nullptr;   // adjoint instead of records
  float *host_out = nullptr;     // host records (copied per level chunk)
  double *host_out64 = nullptr;
  float *dev_out = nullptr;      // device records (written in place)
  double *host_dump = nullptr;   // raw accumulators of one unit
  int dump_level = -1, dump_sub = -1;
};

// Level chunks of one call, as sizes in order.  Without host records:
// chunks of Lc levels.  With records copied to host memory the copy of each
// chunk overlaps the computation of the next, and r = copy time / kernel
// time per level (measured on the previous such call) shapes the chunks:
// r < 1 (kernels dominate): sizes shrink by r towards the end, from m0
// levels at the end, so that the copy left after the last kernel is short
// and every copy fits under the next chunk's kernels; r >= 1 (the copy
// dominates): a first chunk of m0 levels starts the copy engine early.
// Without a measurement: four equal chunks.  No chunk exceeds Lc.
static std::vector<int> level_chunk_sizes(int n, int Lc, bool host_records, double r, int m0) {
  std::vector<int> sz;
  if (n <= 0) return sz;
  auto uniform = [&](int from, int q) {
    for (int l = from; l < n; l += q) sz.push_back(std::min(q, n - l));
  };
  if (!host_records) {
    uniform(0, Lc);
    return sz;
  }
  const int q4 = std::min(Lc, std::max(1, (n + 3) / 4));
  m0 = std::max(1, std::min(m0, q4));
  if (!(r > 0.0) || n < 4) {
    uniform(0, q4);
  } else if (r < 1.0) {
    std::vector<int> back; // last chunk first
    double want = m0;
    int sum = 0;
    while (sum < n) {
      const int c = std::min({Lc, n - sum, std::max(1, (int)std::ceil(want - 1e-9))});
      back.push_back(c);
      sum += c;
      want = want / std::max(r, 0.25);
    }
    sz.assign(back.rbegin(), back.rend());
  } else {
    sz.push_back(m0);
    uniform(m0, std::min(Lc, std::max(m0, (n - m0 + 3) / 4)));
  }
  return sz;
}

// Work-queue order of the units of one batch: most near lines first, ties in
// unit order (two stable 8-bit radix passes on 65535 - bound; bounds above
// 65535 are refused later and sort with 65535).
static void order_by_bound(const int *nb, int n, int *out, std::vector<int> &tmp) {
  tmp.resize(n);
  auto key = [&](int i) { return 65535 - std::min(std::max(nb[i], 0), 65535); };
  int cnt[256];
  std::fill(cnt, cnt + 256, 0);
  for (int i = 0; i < n; ++i) ++cnt[key(i) & 255];
  for (int d = 0, sum = 0; d < 256; ++d) {
    const int c = cnt[d];
    cnt[d] = sum;
    sum += c;
  }
  for (int i = 0; i < n; ++i) tmp[cnt[key(i) & 255]++] = i;
  std::fill(cnt, cnt + 256, 0);
  for (int i = 0; i < n; ++i) ++cnt[key(i) >> 8];
  for (int d = 0, sum = 0; d < 256; ++d) {
    const int c = cnt[d];
    cnt[d] = sum;
    sum += c;
  }
  for (int i = 0; i < n; ++i) out[cnt[key(tmp[i]) >> 8]++] = tmp[i];
}

// What one call of run_levels decides before it launches anything: the
// precision form, the chunks of levels and their fine-kernel plans, the work
// order of the units, the device tables.
struct CallPlan {
  int nsub = 0, C = 0, chi = MARFA_CHI_NONE;
  int64_t N = 0;
  bool f64 = false, adj = false, host_records = false, two = false;
  Consts cst{};
  double sscale = 1.0;                 // FP32c intensity scale
  size_t elem = 4;                     // bytes per accumulator
  int Lc = 0, UB = 0;                  // levels per chunk, units per fine/cascade batch
  int n_chunks = 0;
  std::vector<int> lb;                 // chunk c holds levels [lb[c], lb[c + 1])
  std::vector<int> order;              // work-queue order of the units of every batch
  std::vector<FineChunk> fine;         // fine-kernel launch plan per chunk
  std::vector<double> margin;          // window margin per level
  std::vector<long long> sig;          // the launch plan, for graph replays
  double *d_s = nullptr, *d_e = nullptr;       // device window table
  int64_t *d_lo = nullptr, *d_hi = nullptr;
  int *d_sc0 = nullptr;
  int64_t *d_cb = nullptr, *d_ce = nullptr;    // device far-chunk table
  int *d_cs = nullptr;
  LevelConst *d_lv = nullptr;
  double *d_margin = nullptr;
};

// Timing events of every kernel family of one call, resolved by
// marfa_last_timings (none inside a graph capture).
struct Timeline {
  marfa_ctx *ctx;
  bool off;
  size_t used = 0;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> copies; // record copies
  cudaEvent_t next() {
    if (off) return nullptr;
    if (used == ctx->events.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
      ctx->events.push_back(e);
    }
    return ctx->events[used++];
  }
  void mark(int fam, cudaEvent_t a, cudaEvent_t b) { ctx->marks.push_back({fam, {a, b}}); }
};

// The per-chunk device buffers: set 1 is the second stream's copy.
struct ChunkBufs {
  DevBuf *nus, *gen, *hot, *rank, *snu, *sidx, *far, *fold, *scr, *gstage, *vbuf, *queue;
};
static ChunkBufs chunk_bufs(marfa_ctx *ctx, int set) {
  if (set)
    return {&ctx->b2_nus, &ctx->b2_gen, &ctx->b2_hot, &ctx->b2_rank, &ctx->b2_snu, &ctx->b2_sidx, &ctx->b2_far,
            &ctx->b2_fold, &ctx->b2_scr, &ctx->b2_gstage, &ctx->b2_vbuf, &ctx->b2_queue};
  return {&ctx->b_nus, &ctx->b_gen, &ctx->b_hot, &ctx->b_rank, &ctx->b_snu, &ctx->b_sidx, &ctx->b_far, &ctx->b_fold,
          &ctx->b_scr, &ctx->b_gstage, &ctx->b_vbuf, &ctx->b_queue};
}

// Precision constants, the memory plan (levels per chunk, units per batch)
// and the chunks of levels; creates the streams and events the call needs.
static int plan_call(marfa_ctx *ctx, const marfa_run *run, int n_levels, const Outputs &o, const Plan &pl,
                     CallPlan &cp) {
  const int nsub = pl.n_sub;
  const int64_t N = ctx->n_lines;
  const bool f64 = run->precision == MARFA_PREC_FP64;
  const int C = (int)pl.chunk_sub.size();
  cp.nsub = nsub;
  cp.N = N;
  cp.f64 = f64;
  cp.C = C;
  cp.chi = run->mol_code == 2 ? run->chi : MARFA_CHI_NONE; // CO2-only factors
  cp.cst = make_consts();

  // FP32-compensated form: scale intensities by 2^E so that every partial
  // sum stays far from the float underflow and overflow limits.
  double sscale = 1.0;
  if (!f64) {
    const double top = std::max(ctx->smax, 1e-300) * 3e7;
    int E = 60 - (int)std::ceil(std::log2(top));
    E = std::max(-100, std::min(120, E));
    sscale = std::ldexp(1.0, E);
  }

  // memory plan: levels per chunk and units per fine/cascade batch
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  const bool adj = o.vjp != nullptr;
  const size_t per_level = (size_t)N * (8 + sizeof(LineGen) + (f64 ? sizeof(Hot64) : sizeof(Hot32)) + 8 + 8 + 4 +
                                        (adj ? sizeof(LineAux) : 0)) +
                           (size_t)C * NFAR * 8 + (size_t)nsub * NT * (o.dev_out || adj ? 0 : 8) +
                           (o.host_out64 ? (size_t)nsub * NT * 8 : 0);
  const size_t reuse = ctx->b_nus.cap + ctx->b_gen.cap + ctx->b_hot.cap + ctx->b_rank.cap + ctx->b_snu.cap +
                       ctx->b_sidx.cap + ctx->b_far.cap + ctx->b_out.cap + ctx->b_out64.cap;
  const size_t budget = (size_t)((double)(free_b + reuse) * 0.55);
  int Lc = (int)std::max<size_t>(1, std::min<size_t>((size_t)n_levels, budget / std::max<size_t>(per_level, 1)));
  const size_t elem = f64 ? 8 : 4;
  const size_t unit_bytes = (size_t)SCR_STRIDE * elem * (adj ? 2 : 1); // + gradient scratch
  const size_t scr_budget = std::max<size_t>(unit_bytes, std::min<size_t>((size_t)4 << 30, (free_b + ctx->b_scr.cap) / 5));
  int UB = (int)std::max<size_t>(1, std::min<size_t>((size_t)Lc * nsub, scr_budget / unit_bytes));
  if (o.graph && o.graph->replay) { // the captured chunking
    Lc = o.graph->Lc;
    UB = o.graph->UB;
  }
  // host records: chunks of levels (level_chunk_sizes), so that the copy of
  // each overlaps the computation of the next
  const bool host_records = o.host_out != nullptr && !adj;
  const bool two = host_records && !o.host_out64 && !o.host_dump && !o.graph && n_levels >= 2;
  if (two) { // two buffer sets in the same memory
    Lc = std::max(1, Lc / 2);
    UB = std::max(1, UB / 2);
  }
  if (host_records && !ctx->sm_count)
    CK(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device), "device attribute");
  // chunk boundaries: chunk c holds levels [lb[c], lb[c + 1])
  const int m0 = (2 * std::max(ctx->sm_count, 1) + nsub - 1) / nsub; // two blocks per SM at least
  const double r_copy = ctx->rec_compute_ms > 0.0 ? ctx->rec_copy_ms / ctx->rec_compute_ms : 0.0;
  const std::vector<int> csz = level_chunk_sizes(n_levels, Lc, host_records, r_copy, m0);
  std::vector<int> lb(1, 0);
  for (int c : csz) lb.push_back(lb.back() + c);
  const int n_chunks = (int)csz.size();
  if (host_records) {
    // buffers keep the planned chunk size Lc (no chunk exceeds it), so that a
    // changed schedule on a later call reallocates nothing
    UB = std::min(UB, *std::max_element(csz.begin(), csz.end()) * nsub);
    if (!ctx->copy_stream) CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "copy stream");
    for (int h = 0; h < 2; ++h) {
      if (!ctx->rec_ready[h]) CK(cudaEventCreateWithFlags(&ctx->rec_ready[h], cudaEventDisableTiming), "event");
      if (!ctx->rec_copied[h]) CK(cudaEventCreateWithFlags(&ctx->rec_copied[h], cudaEventDisableTiming), "event");
    }
  }
  if (two) {
    if (!ctx->stream2) CK(cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking), "second stream");
    if (!ctx->fork_ev) CK(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming), "event");
    if (!ctx->join_ev) CK(cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming), "event");
  }
  cp.sscale = sscale;
  cp.adj = adj;
  cp.elem = elem;
  cp.Lc = Lc;
  cp.UB = UB;
  cp.host_records = host_records;
  cp.two = two;
  cp.lb = lb;
  cp.n_chunks = n_chunks;
  return MARFA_OK;
}

// The call's device buffers (grown, never shrunk), the addresses of its
// window and chunk tables and the window margin of every level.
static int alloc_buffers(marfa_ctx *ctx, int n_levels, const double *P, const Outputs &o, CallPlan &cp) {
  const int nsub = cp.nsub, C = cp.C, Lc = cp.Lc, UB = cp.UB;
  const int64_t N = cp.N;
  const bool f64 = cp.f64, adj = cp.adj, two = cp.two;
  const size_t elem = cp.elem;
  CK(ensure(ctx, ctx->b_nus, (size_t)Lc * N * 8), "alloc nus");
  CK(ensure(ctx, ctx->b_gen, (size_t)Lc * N * sizeof(LineGen)), "alloc gen");
  CK(ensure(ctx, ctx->b_hot, (size_t)Lc * N * (f64 ? sizeof(Hot64) : sizeof(Hot32))), "alloc hot");
  CK(ensure(ctx, ctx->b_rank, (size_t)Lc * N * 8), "alloc rank");
  CK(ensure(ctx, ctx->b_snu, (size_t)Lc * N * 8), "alloc snu");
  CK(ensure(ctx, ctx->b_sidx, (size_t)Lc * N * 4), "alloc sidx");
  CK(ensure(ctx, ctx->b_far, (size_t)Lc * std::max(C, 1) * NFAR * 8), "alloc far");
  CK(ensure(ctx, ctx->b_fold, (size_t)Lc * nsub * NFAR * 8), "alloc far sums");
  CK(ensure(ctx, ctx->b_scr, (size_t)UB * SCR_STRIDE * elem), "alloc scratch");
  if (two) {
    CK(ensure(ctx, ctx->b2_nus, ctx->b_nus.cap), "alloc nus");
    CK(ensure(ctx, ctx->b2_gen, ctx->b_gen.cap), "alloc gen");
    CK(ensure(ctx, ctx->b2_hot, ctx->b_hot.cap), "alloc hot");
    CK(ensure(ctx, ctx->b2_rank, ctx->b_rank.cap), "alloc rank");
    CK(ensure(ctx, ctx->b2_snu, ctx->b_snu.cap), "alloc snu");
    CK(ensure(ctx, ctx->b2_sidx, ctx->b_sidx.cap), "alloc sidx");
    CK(ensure(ctx, ctx->b2_far, ctx->b_far.cap), "alloc far");
    CK(ensure(ctx, ctx->b2_fold, ctx->b_fold.cap), "alloc far sums");
    CK(ensure(ctx, ctx->b2_scr, ctx->b_scr.cap), "alloc scratch");
  }
  if (adj) {
    CK(ensure(ctx, ctx->b_gscr, (size_t)UB * SCR_STRIDE * 8), "alloc gradient scratch");
    CK(ensure(ctx, ctx->b_aux, (size_t)Lc * N * sizeof(LineAux)), "alloc line partials");
  }
  CK(ensure(ctx, ctx->b_lv, (size_t)n_levels * sizeof(LevelConst)), "alloc levels");
  CK(ensure(ctx, ctx->b_margin, (size_t)n_levels * 8), "alloc margin");
  if (!o.dev_out && !adj) CK(ensure(ctx, ctx->b_out, (size_t)2 * Lc * nsub * NT * 4), "alloc out");
  if (o.host_out64) CK(ensure(ctx, ctx->b_out64, (size_t)Lc * nsub * NT * 8), "alloc out64");
  if (o.host_dump) CK(ensure(ctx, ctx->b_dump, (size_t)(NT + 3 * NCELLS) * 8), "alloc dump");
  // window and chunk tables
  const size_t win_bytes = (size_t)nsub * (8 + 8 + 8 + 8) + (size_t)(nsub + 1) * 4;
  CK(ensure(ctx, ctx->b_win, win_bytes), "alloc windows");
  const size_t chunk_bytes = (size_t)std::max(C, 1) * (4 + 8 + 8);
  CK(ensure(ctx, ctx->b_chunks, chunk_bytes), "alloc chunks");

  char *wb = (char *)ctx->b_win.p;
  double *d_s = (double *)wb;
  double *d_e = d_s + nsub;
  int64_t *d_lo = (int64_t *)(d_e + nsub);
  int64_t *d_hi = d_lo + nsub;
  int *d_sc0 = (int *)(d_hi + nsub);
  char *cb = (char *)ctx->b_chunks.p;
  int64_t *d_cb = (int64_t *)cb;
  int64_t *d_ce = d_cb + std::max(C, 1);
  int *d_cs = (int *)(d_ce + std::max(C, 1));
  std::vector<double> margin(n_levels);
  for (int l = 0; l < n_levels; ++l) {
    const double a = ctx->dmin * P[l], b = ctx->dmax * P[l];
    margin[l] = std::fabs(b - a) + 1e-7 + 1e-12 * std::fabs(ctx->nu.back());
  }
  LevelConst *d_lv = (LevelConst *)ctx->b_lv.p;
  double *d_margin = (double *)ctx->b_margin.p;
  cp.d_s = d_s;
  cp.d_e = d_e;
  cp.d_lo = d_lo;
  cp.d_hi = d_hi;
  cp.d_sc0 = d_sc0;
  cp.d_cb = d_cb;
  cp.d_ce = d_ce;
  cp.d_cs = d_cs;
  cp.margin = std::move(margin);
  cp.d_lv = d_lv;
  cp.d_margin = d_margin;
  return MARFA_OK;
}

// Near-line bound and work order of every unit, the fine kernel's launch
// plan per chunk of levels (with the staging and slot buffers it needs), and
// the signature of the whole launch plan.
static int plan_fine(marfa_ctx *ctx, const marfa_run *run, int n_levels, const double *P, const Plan &pl,
                     CallPlan &cp) {
  const int nsub = cp.nsub, chi = cp.chi, Lc = cp.Lc, UB = cp.UB, n_chunks = cp.n_chunks;
  const int64_t N = cp.N;
  const bool f64 = cp.f64, two = cp.two;
  const size_t elem = cp.elem;
  const std::vector<int> &lb = cp.lb;
  // Near-line bound of every unit, from the unshifted centres: a near line
  // has s - 1 < nu' < s + 11 (the bounds of fine_kernel) and nu' = nu + delta
  // P with delta in [dmin, dmax], so nu lies in (s - 1 - dmax P, s + 11 -
  // dmin P).  The bound sizes the fine kernel's staging and orders its work
  // queue (most lines first) before anything is launched, so that no call
  // waits for the device in the middle of its launches.
  // The bound of a chunk's units uses the chunk's largest pressure (the
  // widest shift range): one count per subinterval and chunk.
  std::vector<int> nbound((size_t)n_levels * nsub), order_all((size_t)n_levels * nsub);
  const double *nu = ctx->nu.data();
  for (int c = 0; c < n_chunks; ++c) {
    const double Pmax = *std::max_element(P + lb[c], P + lb[c + 1]);
    for (int isub = 0; isub < nsub; ++isub) {
      const double lo = pl.s[isub] - 1.0 - std::max(ctx->dmax, 0.0) * Pmax - 1e-6;
      const double hi = pl.s[isub] + DELTA_WV + 1.0 - std::min(ctx->dmin, 0.0) * Pmax + 1e-6;
      int64_t a, b;
      ctx->nu_index.range(lo, N, a, b);
      const int64_t a0 = std::lower_bound(nu + a, nu + b, lo) - nu;
      ctx->nu_index.range(hi, N, a, b);
      const int64_t b0 = std::upper_bound(nu + std::max(a, a0), nu + std::max(b, a0), hi) - nu;
      for (int l = lb[c]; l < lb[c + 1]; ++l) nbound[(size_t)l * nsub + isub] = (int)(b0 - a0);
    }
  }
  std::vector<int> tmp;
  for (int c = 0; c < n_chunks; ++c) {
    const int base = lb[c] * nsub, units = (lb[c + 1] - lb[c]) * nsub;
    for (int u0 = 0; u0 < units; u0 += UB)
      order_by_bound(nbound.data() + base + u0, std::min(UB, units - u0), order_all.data() + base + u0, tmp);
  }
  CK(ensure(ctx, ctx->b_order, order_all.size() * 4), "alloc order");

  // launch plan of the fine kernel per chunk of levels: staged lines per
  // block in shared memory (units with more near lines stage in a global
  // slice of their block), block size, slot rows in shared memory, grid
  std::vector<FineChunk> fchunks;
  size_t gstage_need = 0, vbuf_need = 0;
  for (int c = 0; c < n_chunks; ++c) {
    const int l0 = lb[c], units = (lb[c + 1] - lb[c]) * nsub;
    FineChunk fc;
    fc.max_near = *std::max_element(nbound.begin() + (size_t)l0 * nsub, nbound.begin() + (size_t)l0 * nsub + units);
    if (fc.max_near > 65535) // line indices of one unit are 16-bit in the fine kernel's bin table
      return set_err(ctx, MARFA_E_CAPACITY, "%d lines within 1 cm-1 of one subinterval (at most 65535)",
                     fc.max_near);
    fc.block_threads = fine_block_threads(run->precision, fc.max_near, ctx->tune.small_block_lines,
                                          ctx->tune.fine_pair);
    // on-chip staging up to what the block's shared memory holds beside the
    // kernel's static arrays (each unit then keeps its slot rows on chip
    // when they fit beside its own lines)
    int smem_lines = 0;
    CK(fine_smem_lines(run->precision, chi, fc.block_threads, &smem_lines), "fine shared memory");
    fc.smem_cap = std::max(128, std::min(smem_lines, (fc.max_near + 127) / 128 * 128));
    fc.gstage_cap = fc.max_near > fc.smem_cap ? (fc.max_near + 255) / 256 * 256 : 0;
    fc.gstage_bytes = fc.gstage_cap ? fine_smem_bytes(fc.gstage_cap, f64) : 0;
    CK(fine_plan(run->precision, chi, fc.block_threads, fc.smem_cap, &fc.smem_room, &fc.resident), "fine occupancy");
    gstage_need = std::max(gstage_need, (size_t)fc.resident * fc.gstage_bytes);
    vbuf_need = std::max(vbuf_need, (size_t)fc.resident *
                                        fine_vbuf_elems(std::max(fc.smem_cap, fc.gstage_cap)) * elem);
    fchunks.push_back(fc);
  }
  if (gstage_need) CK(ensure(ctx, ctx->b_gstage, gstage_need), "alloc staging");
  CK(ensure(ctx, ctx->b_vbuf, vbuf_need), "alloc slot buffers");
  CK(ensure(ctx, ctx->b_queue, 256), "alloc queue");
  if (two) {
    if (gstage_need) CK(ensure(ctx, ctx->b2_gstage, gstage_need), "alloc staging");
    CK(ensure(ctx, ctx->b2_vbuf, vbuf_need), "alloc slot buffers");
    CK(ensure(ctx, ctx->b2_queue, 256), "alloc queue");
  }

  // a captured graph replays only the launch plan it was captured with
  std::vector<long long> sig = {Lc, UB, (long long)ctx->alloc_gen};
  sig.insert(sig.end(), lb.begin(), lb.end());
  for (const FineChunk &fc : fchunks)
    sig.insert(sig.end(), {fc.smem_cap, fc.gstage_cap, fc.block_threads, (long long)fc.smem_room, fc.resident});
  cp.order = std::move(order_all);
  cp.fine = std::move(fchunks);
  cp.sig = std::move(sig);
  return MARFA_OK;
}

// The window, chunk, level and order tables, through the pinned staging ring.
static int stage_tables(marfa_ctx *ctx, cudaStream_t st, int n_levels, const Plan &pl,
                        const std::vector<LevelConst> &lv, const CallPlan &cp) {
  const int nsub = cp.nsub, C = cp.C;
  double *d_s = cp.d_s, *d_e = cp.d_e, *d_margin = cp.d_margin;
  int64_t *d_lo = cp.d_lo, *d_hi = cp.d_hi, *d_cb = cp.d_cb, *d_ce = cp.d_ce;
  int *d_sc0 = cp.d_sc0, *d_cs = cp.d_cs;
  LevelConst *d_lv = cp.d_lv;
  const std::vector<double> &margin = cp.margin;
  const std::vector<int> &order_all = cp.order;
  Staging sg{ctx, st};
  const size_t stage_bytes = 4 * Staging::room((size_t)nsub * 8) + Staging::room((size_t)(nsub + 1) * 4) +
                             2 * Staging::room((size_t)C * 8) + Staging::room((size_t)C * 4) +
                             Staging::room((size_t)n_levels * sizeof(LevelConst)) +
                             Staging::room((size_t)n_levels * 8) + Staging::room(order_all.size() * 4);
  CK(sg.begin(stage_bytes), "pinned staging");
  CK(sg.put(d_s, pl.s.data(), nsub * 8), "h2d windows");
  CK(sg.put(d_e, pl.e.data(), nsub * 8), "h2d windows");
  CK(sg.put(d_lo, pl.lo.data(), nsub * 8), "h2d windows");
  CK(sg.put(d_hi, pl.hi.data(), nsub * 8), "h2d windows");
  CK(sg.put(d_sc0, pl.sub_chunk0.data(), (nsub + 1) * 4), "h2d windows");
  CK(sg.put(d_cb, pl.chunk_begin.data(), (size_t)C * 8), "h2d chunks");
  CK(sg.put(d_ce, pl.chunk_end.data(), (size_t)C * 8), "h2d chunks");
  CK(sg.put(d_cs, pl.chunk_sub.data(), (size_t)C * 4), "h2d chunks");
  CK(sg.put(d_lv, lv.data(), n_levels * sizeof(LevelConst)), "h2d levels");
  CK(sg.put(d_margin, margin.data(), n_levels * 8), "h2d margin");
  CK(sg.put(ctx->b_order.p, order_all.data(), order_all.size() * 4), "h2d order");
  CK(sg.end(), "staging event");
  return MARFA_OK;
}

// The launches of chunk c of levels, on its stream: prep (and the adjoint's
// prep), sort, far kernel, then per batch of units the fine kernel and the
// cascade (or the adjoint kernels), and the copy of the chunk's records.
static int launch_chunk(marfa_ctx *ctx, const marfa_run *run, const Outputs &o, const Plan &pl,
                        const CallPlan &cp, int c, cudaStream_t st, Timeline &tl) {
  const int nsub = cp.nsub, C = cp.C, chi = cp.chi, Lc = cp.Lc, UB = cp.UB;
  const int64_t N = cp.N;
  const bool f64 = cp.f64, adj = cp.adj, two = cp.two, host_records = cp.host_records;
  const Consts cst = cp.cst;
  const double sscale = cp.sscale;
  const std::vector<int> &lb = cp.lb;
  const std::vector<FineChunk> &fchunks = cp.fine;
  int *d_sc0 = cp.d_sc0, *d_cs = cp.d_cs;
  int64_t *d_cb = cp.d_cb, *d_ce = cp.d_ce;
  LevelConst *d_lv = cp.d_lv;
  double *d_margin = cp.d_margin;
  const WindowTable win{cp.d_s, cp.d_e, cp.d_lo, cp.d_hi, nsub};
  DeviceLines dl{ctx->d_nu, ctx->d_S, ctx->d_gair, ctx->d_gself, ctx->d_elow, ctx->d_nair, ctx->d_delta, ctx->d_iso, N,
                 ctx->d_S64, ctx->d_gair64};
  auto next_event = [&]() { return tl.next(); };
  auto mark = [&](int fam, cudaEvent_t a, cudaEvent_t b) { tl.mark(fam, a, b); };
  auto &copy_marks = tl.copies;
  const int l0 = lb[c], nl = lb[c + 1] - lb[c];
  // chunk c runs on stream c % 2 with buffer set c % 2 (one of each
  // without host records); chunk c - 2 used the same ones on the same stream
  const int set = two ? (c & 1) : 0;
  const ChunkBufs B = chunk_bufs(ctx, set);
  cudaStream_t cs = set ? ctx->stream2 : st;
  PrepParams pp;
  pp.lines = dl;
  pp.tips = ctx->d_tips;
  pp.n_iso = ctx->n_iso;
  pp.n_temp = ctx->n_temp;
  pp.tgrid = ctx->tgrid;
  pp.lv = d_lv + l0;
  pp.n_levels = nl;
  pp.c = cst;
  pp.sscale = sscale;
  pp.nus = (double *)B.nus->p;
  pp.gen = (LineGen *)B.gen->p;
  pp.hot32 = f64 ? nullptr : (Hot32 *)B.hot->p;
  pp.hot64 = f64 ? (Hot64 *)B.hot->p : nullptr;
  pp.err = ctx->d_err;
  cudaEvent_t e0 = next_event(), e1 = next_event(), e2 = next_event(), e3 = next_event();
  if (e0) cudaEventRecord(e0, cs);
  CK(launch_prep(pp, cs), "prep kernel");
  ctx->launches += 1;
  if (adj) {
    AdjPrepParams ap;
    ap.lines = dl;
    ap.tips = ctx->d_tips;
    ap.n_iso = ctx->n_iso;
    ap.n_temp = ctx->n_temp;
    ap.tgrid = ctx->tgrid;
    ap.lv = pp.lv;
    ap.n_levels = nl;
    ap.c = cst;
    ap.aux = (LineAux *)ctx->b_aux.p;
    CK(launch_adjoint_prep(ap, cs), "adjoint prep kernel");
    ctx->launches += 1;
  }
  if (e1) cudaEventRecord(e1, cs);
  SortParams sp;
  sp.nu = ctx->d_nu;
  sp.nus = pp.nus;
  sp.margin = d_margin + l0;
  sp.n = N;
  sp.n_levels = nl;
  sp.rank = (int64_t *)B.rank->p;
  sp.snu = (double *)B.snu->p;
  sp.sidx = (int *)B.sidx->p;
  CK(launch_sort(sp, cs), "sort kernels");
  ctx->launches += 2;
  if (e2) cudaEventRecord(e2, cs);
  FarParams fp;
  fp.nus = pp.nus;
  fp.hot32 = pp.hot32;
  fp.hot64 = pp.hot64;
  fp.gen = pp.gen;
  fp.lv = pp.lv;
  fp.win = win;
  fp.chunk_sub = d_cs;
  fp.chunk_begin = d_cb;
  fp.chunk_end = d_ce;
  fp.n_chunks = C;
  fp.n_levels = nl;
  fp.n_lines = N;
  fp.cutoff = run->cutoff;
  fp.sscale = sscale;
  fp.shape = run->shape;
  fp.c = cst;
  fp.out = (double *)B.far->p;
  CK(launch_far(fp, run->precision, chi, cs), "far kernel");
  if (C > 0) {
    ctx->launches += 1;
    ctx->far_launches += 1;
  }
  if (e3) cudaEventRecord(e3, cs);
  // far sums per (level, subinterval, grid-0 position), read by the cascade
  double *fold = (double *)B.fold->p;
  CK(launch_far_fold(fp.out, d_sc0, C, nsub, nl, fold, cs), "far sums");
  ctx->launches += 1;
  mark(0, e0, e1);
  mark(1, e1, e2);
  mark(2, e2, e3);

  const int half = c & 1;
  float *out_base = o.dev_out ? o.dev_out : (float *)ctx->b_out.p + (size_t)half * Lc * nsub * NT;
  // the half written now was copied out two chunks ago
  if (host_records && c >= 2) CK(cudaStreamWaitEvent(cs, ctx->rec_copied[half], 0), "wait copy");
  const int out_level0 = o.dev_out ? l0 : 0;
  const int units = nl * nsub;
  // near-line counts of this chunk's units size the fine kernel's staging
  FineParams fn;
  fn.snu = sp.snu;
  fn.sidx = sp.sidx;
  fn.gen = pp.gen;
  fn.lv = pp.lv;
  fn.win = win;
  fn.n_lines = N;
  fn.cutoff = run->cutoff;
  fn.sscale = sscale;
  fn.shape = run->shape;
  fn.c = cst;
  fn.scratch = B.scr->p;
  fn.err = ctx->d_err;
  const FineChunk &fc = fchunks[c];
  const int max_near = fc.max_near;
  fn.smem_cap = fc.smem_cap;
  fn.gstage_cap = fc.gstage_cap;
  fn.gstage_bytes = fc.gstage_bytes;
  fn.gstage = fc.gstage_cap ? B.gstage->p : nullptr;
  fn.block_threads = fc.block_threads;
  fn.smem_room = fc.smem_room;
  const int resident = fc.resident;
  fn.vbuf_cap = std::max(fn.smem_cap, fn.gstage_cap);
  fn.vbuf_stride = fine_vbuf_elems(fn.vbuf_cap);
  fn.vbuf = B.vbuf->p;
  fn.queue = (int *)B.queue->p;
  fn.coop_k = ctx->tune.coop_k;
  const int UBc = UB;
  for (int u0 = 0; u0 < units; u0 += UBc) {
    const int nu_ = std::min(UBc, units - u0);
    fn.unit0 = u0;
    fn.n_units = nu_;
    fn.order = (const int *)ctx->b_order.p + (size_t)l0 * nsub + u0;
    fn.grid = std::min(resident, nu_);
    cudaEvent_t f0 = next_event(), f1 = next_event(), f2 = next_event();
    if (f0) cudaEventRecord(f0, cs);
    CK(cudaMemsetAsync(fn.queue, 0, sizeof(int), cs), "memset queue");
    CK(launch_fine(fn, run->precision, chi, cs), "fine kernel");
    ctx->launches += 1;
    if (f1) cudaEventRecord(f1, cs);
    if (adj) {
      CascadeAdjParams ca;
      ca.scratch = (const double *)B.scr->p;
      ca.far = fp.out;
      ca.fold = fold;
      ca.sub_chunk0 = d_sc0;
      ca.lv = pp.lv;
      ca.n_chunks = C;
      ca.n_sub = nsub;
      ca.unit0 = u0;
      ca.n_units = nu_;
      ca.level_out0 = l0;
      ca.target = run->target;
      ca.cot = o.vjp->cot;
      ca.gscratch = (double *)ctx->b_gscr.p;
      CK(launch_cascade_adjoint(ca, cs), "cascade adjoint kernel");
      AdjointParams ad;
      ad.snu = sp.snu;
      ad.sidx = sp.sidx;
      ad.nus = pp.nus;
      ad.gen = pp.gen;
      ad.aux = (const LineAux *)ctx->b_aux.p;
      ad.lv = pp.lv;
      ad.win = win;
      ad.sub_chunk0 = d_sc0;
      ad.chunk_begin = d_cb;
      ad.chunk_end = d_ce;
      ad.max_chunks = pl.max_chunks;
      ad.n_lines = N;
      ad.unit0 = u0;
      ad.n_units = nu_;
      ad.level_out0 = l0;
      ad.cutoff = run->cutoff;
      ad.c = cst;
      ad.gscratch = (const double *)ctx->b_gscr.p;
      ad.dS = o.vjp->dS;
      ad.dgair = o.vjp->dgair;
      ad.dT = o.vjp->dT;
      ad.dP = o.vjp->dP;
      CK(launch_line_adjoint(ad, chi, std::min(64, (max_near + 255) / 256), cs), "line adjoint kernels");
      ctx->launches += 2 + (pl.max_chunks > 0 ? 1 : 0);
      if (f2) cudaEventRecord(f2, cs);
      mark(3, f0, f1);
      mark(4, f1, f2);
      continue;
    }
    CascadeParams cp;
    cp.scratch = B.scr->p;
    cp.far = fp.out;
    cp.fold = fold;
    cp.sub_chunk0 = d_sc0;
    cp.lv = pp.lv;
    cp.n_chunks = C;
    cp.n_sub = nsub;
    cp.unit0 = u0;
    cp.n_units = nu_;
    cp.level_out0 = out_level0;
    cp.inv_sscale = 1.0 / sscale;
    cp.target = run->target;
    cp.out = out_base;
    cp.out64 = o.host_out64 ? (double *)ctx->b_out64.p : nullptr;
    cp.dump = nullptr;
    cp.dump_unit = -1;
    if (o.host_dump && o.dump_level >= l0 && o.dump_level < l0 + nl) {
      cp.dump = (double *)ctx->b_dump.p;
      cp.dump_unit = (o.dump_level - l0) * nsub + o.dump_sub;
    }
    CK(launch_cascade(cp, run->precision, cs), "cascade kernel");
    ctx->launches += cp.dump ? 2 : 1;
    if (f2) cudaEventRecord(f2, cs);
    mark(3, f0, f1);
    mark(4, f1, f2);
  }
  if (host_records) {
    CK(cudaEventRecord(ctx->rec_ready[half], cs), "event");
    CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->rec_ready[half], 0), "wait records");
    cudaEvent_t c0 = next_event(), c1 = next_event();
    if (c0) cudaEventRecord(c0, ctx->copy_stream);
    CK(cudaMemcpyAsync(o.host_out + (size_t)l0 * nsub * NT, out_base, (size_t)nl * nsub * NT * 4,
                       cudaMemcpyDeviceToHost, ctx->copy_stream), "d2h records");
    if (c1) cudaEventRecord(c1, ctx->copy_stream);
    if (c0 && c1) copy_marks.push_back({c0, c1});
    CK(cudaEventRecord(ctx->rec_copied[half], ctx->copy_stream), "event");
  }
  if (o.host_out64)
    CK(cudaMemcpyAsync(o.host_out64 + (size_t)l0 * nsub * NT, ctx->b_out64.p, (size_t)nl * nsub * NT * 8,
                       cudaMemcpyDeviceToHost, cs), "d2h records64");
  return MARFA_OK;
}

// The whole computation for a flat list of levels: plan, tables, then the
// chunks of levels (on two streams when the records go to the host), then
// the end of the call (graph instantiation, or synchronisation, the timing
// of the record copies for the next call's chunks and the device status).
int run_levels(marfa_ctx *ctx, const marfa_run *run, int n_levels, const double *P,
               const double *T, const double *dens, const Outputs &o, cudaStream_t st) {
  int rc = check_run(ctx, run);
  if (rc) return rc;
  if (n_levels < 1 || !P || !T || !dens) return set_err(ctx, MARFA_E_ARG, "no levels");
  Plan pl;
  if ((rc = make_plan(ctx, run, pl))) return rc;
  std::vector<LevelConst> lv;
  if ((rc = build_levels(ctx, n_levels, P, T, dens, lv))) return rc;
  if (pl.n_sub == 0) return MARFA_OK;
  CallPlan cp;
  if ((rc = plan_call(ctx, run, n_levels, o, pl, cp))) return rc;
  if ((rc = alloc_buffers(ctx, n_levels, P, o, cp))) return rc;
  if ((rc = plan_fine(ctx, run, n_levels, P, pl, cp))) return rc;
  if ((rc = stage_tables(ctx, st, n_levels, pl, lv, cp))) return rc;
  const int Lc = cp.Lc, UB = cp.UB, n_chunks = cp.n_chunks;
  const bool two = cp.two, host_records = cp.host_records;
  const std::vector<long long> &sig = cp.sig;
  if (o.graph && o.graph->replay) {
    if (sig != o.graph->sig)
      return set_err(ctx, MARFA_E_ARG, "the graph was captured for another launch plan (line buffers grown or "
                                       "near-line counts changed): create a new graph");
    CK(cudaGraphLaunch(o.graph->exec, st), "graph launch");
    ctx->marks.clear();
    ctx->launches = o.graph->launches;
    ctx->far_launches = 0;
    return MARFA_OK;
  }
  if (o.graph) {
    o.graph->sig = sig;
    o.graph->Lc = Lc;
    o.graph->UB = UB;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "begin capture");
  }
  CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st), "memset err");

  // timing events of every kernel family, resolved by marfa_last_timings
  ctx->marks.clear();
  ctx->launches = 0;
  ctx->far_launches = 0;
  Timeline tl{ctx, o.graph != nullptr, 0, {}};
  cudaEvent_t ev_begin = tl.next();
  if (ev_begin) cudaEventRecord(ev_begin, st);
  if (two) { // the second stream starts after the tables and the error flag
    CK(cudaEventRecord(ctx->fork_ev, st), "event");
    CK(cudaStreamWaitEvent(ctx->stream2, ctx->fork_ev, 0), "fork");
  }
  for (int c = 0; c < n_chunks; ++c)
    if ((rc = launch_chunk(ctx, run, o, pl, cp, c, st, tl))) return rc;
  if (two) { // join the second stream
    CK(cudaEventRecord(ctx->join_ev, ctx->stream2), "event");
    CK(cudaStreamWaitEvent(st, ctx->join_ev, 0), "join");
  }
  cudaEvent_t ev_end = tl.next();
  if (ev_end) cudaEventRecord(ev_end, st);
  if (ev_begin && ev_end) tl.mark(5, ev_begin, ev_end);
  if (o.host_dump)
    CK(cudaMemcpyAsync(o.host_dump, ctx->b_dump.p, (size_t)(NT + 3 * NCELLS) * 8, cudaMemcpyDeviceToHost, st),
       "d2h dump");
  if (o.graph) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamEndCapture(st, &g), "end capture");
    const cudaError_t e = cudaGraphInstantiate(&o.graph->exec, g, 0);
    cudaGraphDestroy(g);
    CK(e, "graph instantiate");
    o.graph->launches = ctx->launches;
    return MARFA_OK;
  }
  if (o.dev_out) return MARFA_OK; // asynchronous path: caller synchronises
  CK(cudaStreamSynchronize(st), "stream sync");
  if (host_records) {
    CK(cudaStreamSynchronize(ctx->copy_stream), "copy stream sync");
    // kernel and copy time per level, for the chunks of the next call (the
    // kernels' time from the call's first to its last kernel: the chunks'
    // kernels overlap on two streams)
    double kms = 0.0, cms = 0.0;
    float ms = 0.f;
    for (auto &m : ctx->marks)
      if (m.first == 5 && cudaEventElapsedTime(&ms, m.second.first, m.second.second) == cudaSuccess) kms += ms;
    for (auto &m : tl.copies)
      if (cudaEventElapsedTime(&ms, m.first, m.second) == cudaSuccess) cms += ms;
    if (kms > 0.0 && cms > 0.0 && tl.copies.size() == (size_t)n_chunks) {
      ctx->rec_compute_ms = kms / n_levels;
      ctx->rec_copy_ms = cms / n_levels;
    }
  }
  int herr = 0;
  CK(cudaMemcpy(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost), "d2h err");
  if (herr) return set_err(ctx, herr, "device reported status %d (isotopologue or temperature outside tables)", herr);
  return MARFA_OK;
}

int total_levels(marfa_ctx *ctx, int n_profiles, const int *counts, int &total) {
  total = 0;
  if (n_profiles < 1 || !counts) return set_err(ctx, MARFA_E_ARG, "no profiles");
  for (int i = 0; i < n_profiles; ++i) {
    if (counts[i] < 1) return set_err(ctx, MARFA_E_ARG, "profile %d has no levels", i);
    if (counts[i] > 200) return set_err(ctx, 6, "profile %d has %d levels > 200", i, counts[i]);
    total += counts[i];
  }
  return MARFA_OK;
}

} // namespace

extern "C" {

int marfa_num_subintervals(double start_wv, double end_wv) {
  int n = 0;
  double s = start_wv;
  while (s < end_wv) {
    ++n;
    s = s + DELTA_WV;
  }
  return n;
}

int marfa_record_number(double start_wv, int isub) {
  double s = start_wv;
  for (int i = 0; i < isub; ++i) s = s + DELTA_WV;
  return (int)((s + 1.0) / 10.0);
}

int marfa_plan_windows(const double *nu, int64_t n_lines, double start_wv, double end_wv, double cutoff,
                       int64_t *lo, int64_t *hi) {
  if (!nu || n_lines < 1 || !lo || !hi) return MARFA_E_ARG;
  try {
    std::vector<double> ss, se;
    std::vector<int64_t> l, h;
    int bad = -1;
    const int rc = plan_windows(nu, n_lines, start_wv, end_wv, cutoff, ss, se, l, h, bad);
    if (rc) return rc;
    for (size_t i = 0; i < l.size(); ++i) {
      lo[i] = l[i];
      hi[i] = h[i];
    }
    return MARFA_OK;
  } catch (...) {
    return MARFA_E_NOMEM;
  }
}

int marfa_ctx_create(const marfa_line_record *lines, int64_t n_lines, const double *tips, int n_iso,
                     int n_temp, int device, marfa_ctx **out) {
  if (!out) return MARFA_E_ARG;
  *out = nullptr;
  if (!lines || n_lines < 1 || !tips || n_iso < 1 || n_temp < 139 || n_lines > 2000000000LL)
    return MARFA_E_ARG;
  marfa_ctx *ctx = new (std::nothrow) marfa_ctx();
  if (!ctx) return MARFA_E_NOMEM;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    delete ctx;
    return MARFA_E_NODEVICE;
  }
  if (device < 0 || device >= ndev) {
    delete ctx;
    return MARFA_E_ARG;
  }
  ctx->device = device;
  ctx->n_lines = n_lines;
  ctx->n_iso = n_iso;
  ctx->n_temp = n_temp;
  ctx->nu.resize(n_lines);
  std::vector<float> S(n_lines), ga(n_lines), gs(n_lines), el(n_lines), na(n_lines), de(n_lines);
  std::vector<int> iso(n_lines);
  ctx->dmin = 1e300;
  ctx->dmax = -1e300;
  for (int64_t i = 0; i < n_lines; ++i) {
    const marfa_line_record &r = lines[i];
    if (!std::isfinite(r.nu) || (i > 0 && r.nu < lines[i - 1].nu)) {
      delete ctx;
      return MARFA_E_UNSORTED;
    }
    ctx->nu[i] = r.nu;
    S[i] = r.S;
    ga[i] = r.gamma_air;
    gs[i] = r.gamma_self;
    el[i] = r.e_lower;
    na[i] = r.n_air;
    de[i] = r.delta_air;
    iso[i] = r.joint_mol_iso / 100;
    ctx->smax = std::max(ctx->smax, (double)std::fabs(r.S));
    ctx->dmin = std::min(ctx->dmin, (double)r.delta_air);
    ctx->dmax = std::max(ctx->dmax, (double)r.delta_air);
  }
  ctx->nu_index.build(ctx->nu);
  int rc = MARFA_OK;
  auto fail = [&](cudaError_t e, const char *w) {
    rc = cuda_fail(ctx, e, w);
    return rc;
  };
  cudaError_t e;
  if ((e = cudaSetDevice(device)) != cudaSuccess) fail(e, "cudaSetDevice");
  if (!rc && (e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess)
    fail(e, "stream");
  const size_t nb8 = (size_t)n_lines * 8, nb4 = (size_t)n_lines * 4;
  void **ptrs[] = {(void **)&ctx->d_nu, (void **)&ctx->d_S, (void **)&ctx->d_gair, (void **)&ctx->d_gself,
                   (void **)&ctx->d_elow, (void **)&ctx->d_nair, (void **)&ctx->d_delta, (void **)&ctx->d_iso};
  const void *src[] = {ctx->nu.data(), S.data(), ga.data(), gs.data(), el.data(), na.data(), de.data(), iso.data()};
  for (int k = 0; k < 8 && !rc; ++k) {
    const size_t nb = k == 0 ? nb8 : nb4;
    if ((e = cudaMalloc(ptrs[k], nb)) != cudaSuccess) fail(e, "alloc lines");
    else if ((e = cudaMemcpy(*ptrs[k], src[k], nb, cudaMemcpyHostToDevice)) != cudaSuccess) fail(e, "h2d lines");
  }
  if (!rc && (e = cudaMalloc(&ctx->d_tips, (size_t)n_iso * n_temp * 8)) != cudaSuccess) fail(e, "alloc tips");
  if (!rc && (e = cudaMemcpy(ctx->d_tips, tips, (size_t)n_iso * n_temp * 8, cudaMemcpyHostToDevice)) != cudaSuccess)
    fail(e, "h2d tips");
  if (!rc && (e = cudaMalloc(&ctx->d_err, sizeof(int))) != cudaSuccess) fail(e, "alloc err");
  if (rc) {
    int code = rc;
    marfa_ctx_destroy(ctx);
    return code;
  }
  *out = ctx;
  return MARFA_OK;
}

void marfa_ctx_destroy(marfa_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->stream2) cudaStreamSynchronize(ctx->stream2);
  void *ps[] = {ctx->d_nu, ctx->d_S, ctx->d_gair, ctx->d_gself, ctx->d_elow, ctx->d_nair, ctx->d_delta,
                ctx->d_iso, ctx->d_tips, ctx->d_err, ctx->d_S64, ctx->d_gair64};
  for (void *p : ps)
    if (p) cudaFree(p);
  DevBuf *bs[] = {&ctx->b_nus, &ctx->b_gen, &ctx->b_hot, &ctx->b_rank, &ctx->b_snu, &ctx->b_sidx, &ctx->b_far, &ctx->b_fold,
                  &ctx->b_scr, &ctx->b_lv, &ctx->b_margin, &ctx->b_win, &ctx->b_chunks, &ctx->b_out,
                  &ctx->b_out64, &ctx->b_dump, &ctx->b_count, &ctx->b_gstage, &ctx->b_aux,
                  &ctx->b_gscr, &ctx->b_cot, &ctx->b_grad, &ctx->b_vbuf, &ctx->b_queue, &ctx->b_order, &ctx->b_tune,
                  &ctx->b2_nus, &ctx->b2_gen, &ctx->b2_hot, &ctx->b2_rank, &ctx->b2_snu, &ctx->b2_sidx,
                  &ctx->b2_far, &ctx->b2_fold, &ctx->b2_scr, &ctx->b2_gstage, &ctx->b2_vbuf, &ctx->b2_queue};
  for (DevBuf *b : bs) release(*b);
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  for (int h = 0; h < 2; ++h) {
    if (ctx->rec_ready[h]) cudaEventDestroy(ctx->rec_ready[h]);
    if (ctx->rec_copied[h]) cudaEventDestroy(ctx->rec_copied[h]);
  }
  for (int i = 0; i < marfa_ctx::NPIN; ++i) {
    if (ctx->pinned[i]) cudaFreeHost(ctx->pinned[i]);
    if (ctx->pinned_ev[i]) cudaEventDestroy(ctx->pinned_ev[i]);
  }
  for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
  if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char *marfa_last_error(const marfa_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int marfa_compute_batched(marfa_ctx *ctx, const marfa_run *run, int n_profiles, const int *level_counts,
                          const double *pressure, const double *temperature, const double *density,
                          float *out, double *out64) {
  if (!ctx) return MARFA_E_ARG;
  if (!out) return set_err(ctx, MARFA_E_ARG, "out is null");
  int total = 0, rc = total_levels(ctx, n_profiles, level_counts, total);
  if (rc) return rc;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MARFA_E_CUDA, "cudaSetDevice");
  Outputs o;
  o.host_out = out;
  o.host_out64 = out64;
  try {
    return run_levels(ctx, run, total, pressure, temperature, density, o, ctx->stream);
  } catch (...) {
    return set_err(ctx, MARFA_E_NOMEM, "host allocation failed");
  }
}

int marfa_compute(marfa_ctx *ctx, const marfa_run *run, const double *pressure, const double *temperature,
                  const double *density, int n_levels, float *out, double *out64) {
  return marfa_compute_batched(ctx, run, 1, &n_levels, pressure, temperature, density, out, out64);
}

int marfa_compute_device(marfa_ctx *ctx, const marfa_run *run, int n_profiles, const int *level_counts,
                         const double *pressure, const double *temperature, const double *density,
                         float *device_out, void *stream) {
  if (!ctx) return MARFA_E_ARG;
  if (!device_out) return set_err(ctx, MARFA_E_ARG, "device_out is null");
  int total = 0, rc = total_levels(ctx, n_profiles, level_counts, total);
  if (rc) return rc;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MARFA_E_CUDA, "cudaSetDevice");
  Outputs o;
  o.dev_out = device_out;
  try {
    return run_levels(ctx, run, total, pressure, temperature, density, o,
                      stream ? (cudaStream_t)stream : ctx->stream);
  } catch (...) {
    return set_err(ctx, MARFA_E_NOMEM, "host allocation failed");
  }
}

int marfa_ctx_set_line_params(marfa_ctx *ctx, const double *S, const double *gamma_air) {
  if (!ctx) return MARFA_E_ARG;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MARFA_E_CUDA, "cudaSetDevice");
  CK(cudaStreamSynchronize(ctx->stream), "stream sync");
  const size_t nb = (size_t)ctx->n_lines * 8;
  auto put = [&](double *&dst, const double *src) -> int {
    if (!src) {
      if (dst) cudaFree(dst);
      dst = nullptr;
      return MARFA_OK;
    }
    for (int64_t i = 0; i < ctx->n_lines; ++i)
      if (!std::isfinite(src[i])) return set_err(ctx, MARFA_E_ARG, "line %lld: non-finite value", (long long)i);
    if (!dst) CK(cudaMalloc(&dst, nb), "alloc line overrides");
    CK(cudaMemcpy(dst, src, nb, cudaMemcpyHostToDevice), "h2d line overrides");
    return MARFA_OK;
  };
  int rc = put(ctx->d_S64, S);
  if (!rc) rc = put(ctx->d_gair64, gamma_air);
  if (rc) return rc;
  // the intensity scale of the FP32-compensated form follows the largest S
  double smax = 0.0;
  if (S) {
    for (int64_t i = 0; i < ctx->n_lines; ++i) smax = std::max(smax, std::fabs(S[i]));
  } else {
    std::vector<float> Sf(ctx->n_lines);
    CK(cudaMemcpy(Sf.data(), ctx->d_S, (size_t)ctx->n_lines * 4, cudaMemcpyDeviceToHost), "d2h S");
    for (float v : Sf) smax = std::max(smax, (double)std::fabs(v));
  }
  ctx->smax = smax;
  return MARFA_OK;
}

int marfa_vjp(marfa_ctx *ctx, const marfa_run *run, const double *pressure, const double *temperature,
              const double *density, int n_levels, const double *cotangent, double *d_temperature,
              double *d_pressure, double *d_S, double *d_gamma_air) {
  if (!ctx) return MARFA_E_ARG;
  if (!run || !cotangent || !d_temperature || !d_pressure || !d_S || !d_gamma_air)
    return set_err(ctx, MARFA_E_ARG, "null argument");
  if (run->shape != MARFA_SHAPE_VOIGT) return set_err(ctx, MARFA_E_ARG, "the adjoint needs the Voigt shape");
  if (n_levels < 1) return set_err(ctx, MARFA_E_ARG, "no levels");
  if (n_levels > 200) return set_err(ctx, 6, "%d levels > 200", n_levels);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MARFA_E_CUDA, "cudaSetDevice");
  marfa_run r = *run;
  r.precision = MARFA_PREC_FP64;
  int rc = check_run(ctx, &r);
  if (rc) return rc;
  const int nsub = marfa_num_subintervals(r.start_wv, r.end_wv);
  const int64_t N = ctx->n_lines;
  cudaStream_t st = ctx->stream;
  try {
    const size_t ncot = (size_t)n_levels * nsub * NT;
    CK(ensure(ctx, ctx->b_cot, std::max<size_t>(ncot, 1) * 8), "alloc cotangent");
    CK(ensure(ctx, ctx->b_grad, ((size_t)2 * N + 2 * n_levels) * 8), "alloc gradients");
    double *g = (double *)ctx->b_grad.p;
    VjpOut v;
    v.cot = (const double *)ctx->b_cot.p;
    v.dS = g;
    v.dgair = g + N;
    v.dT = g + 2 * N;
    v.dP = g + 2 * N + n_levels;
    if (ncot) CK(cudaMemcpyAsync(ctx->b_cot.p, cotangent, ncot * 8, cudaMemcpyHostToDevice, st), "h2d cotangent");
    CK(cudaMemsetAsync(g, 0, ((size_t)2 * N + 2 * n_levels) * 8, st), "memset gradients");
    Outputs o;
    o.vjp = &v;
    rc = run_levels(ctx, &r, n_levels, pressure, temperature, density, o, st);
    if (rc) return rc;
    CK(cudaMemcpyAsync(d_S, v.dS, (size_t)N * 8, cudaMemcpyDeviceToHost, st), "d2h dS");
    CK(cudaMemcpyAsync(d_gamma_air, v.dgair, (size_t)N * 8, cudaMemcpyDeviceToHost, st), "d2h dgamma");
    CK(cudaMemcpyAsync(d_temperature, v.dT, (size_t)n_levels * 8, cudaMemcpyDeviceToHost, st), "d2h dT");
    CK(cudaMemcpyAsync(d_pressure, v.dP, (size_t)n_levels * 8, cudaMemcpyDeviceToHost, st), "d2h dP");
    CK(cudaStreamSynchronize(st), "stream sync");
    return MARFA_OK;
  } catch (...) {
    return set_err(ctx, MARFA_E_NOMEM, "host allocation failed");
  }
}

struct marfa_graph {
  marfa_ctx *ctx = nullptr;
  marfa_run run{};
  int total = 0;
  float *dev_out = nullptr;
  GraphCtl ctl;
};

int marfa_graph_create(marfa_ctx *ctx, const marfa_run *run, int n_profiles, const int *level_counts,
                       const double *pressure, const double *temperature, const double *density,
                       float *device_out, marfa_graph **out) {
  if (!ctx || !out) return MARFA_E_ARG;
  *out = nullptr;
  if (!run || !device_out) return set_err(ctx, MARFA_E_ARG, "null argument");
  int total = 0, rc = total_levels(ctx, n_profiles, level_counts, total);
  if (rc) return rc;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MARFA_E_CUDA, "cudaSetDevice");
  marfa_graph *g = new (std::nothrow) marfa_graph();
  if (!g) return set_err(ctx, MARFA_E_NOMEM, "host allocation failed");
  g->ctx = ctx;
  g->run = *run;
  g->total = total;
  g->dev_out = device_out;
  try {
    // one eager call allocates every buffer (no allocation may happen while
    // the stream is captured) and computes the records; the second call is
    // captured
    Outputs o;
    o.dev_out = device_out;
    rc = run_levels(ctx, run, total, pressure, temperature, density, o, ctx->stream);
    if (!rc) rc = marfa_synchronize(ctx);
    if (!rc) {
      o.graph = &g->ctl;
      rc = run_levels(ctx, run, total, pressure, temperature, density, o, ctx->stream);
    }
  } catch (...) {
    rc = set_err(ctx, MARFA_E_NOMEM, "host allocation failed");
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(ctx->stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
    cudaGraph_t dead = nullptr; // a failed capture: close it and drop the graph
    cudaStreamEndCapture(ctx->stream, &dead);
    if (dead) cudaGraphDestroy(dead);
  }
  if (rc || !g->ctl.exec) {
    marfa_graph_destroy(g);
    return rc ? rc : set_err(ctx, MARFA_E_CUDA, "graph capture produced no graph");
  }
  g->ctl.replay = true;
  *out = g;
  return MARFA_OK;
}

int marfa_graph_launch(marfa_graph *g, const double *pressure, const double *temperature,
                       const double *density, void *stream) {
  if (!g) return MARFA_E_ARG;
  if (cudaSetDevice(g->ctx->device) != cudaSuccess) return set_err(g->ctx, MARFA_E_CUDA, "cudaSetDevice");
  Outputs o;
  o.dev_out = g->dev_out;
  o.graph = &g->ctl;
  try {
    return run_levels(g->ctx, &g->run, g->total, pressure, temperature, density, o,
                      stream ? (cudaStream_t)stream : g->ctx->stream);
  } catch (...) {
    return set_err(g->ctx, MARFA_E_NOMEM, "host allocation failed");
  }
}

void marfa_graph_destroy(marfa_graph *g) {
  if (!g) return;
  if (g->ctl.exec) cudaGraphExecDestroy(g->ctl.exec);
  delete g;
}

int marfa_autotune(marfa_ctx *ctx, const marfa_run *run, int n_levels, const double *pressure,
                   const double *temperature, const double *density, int *far_chunk, int *coop_k) {
  if (!ctx) return MARFA_E_ARG;
  if (!run || n_levels < 1 || !pressure || !temperature || !density)
    return set_err(ctx, MARFA_E_ARG, "null argument");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MARFA_E_CUDA, "cudaSetDevice");
  // sample: up to sixteen levels spread over the profile, every subinterval
  // (a far-kernel grid of a few levels has too few blocks and favours small
  // chunks that lose on a whole profile)
  constexpr int kSample = 16;
  std::vector<int> pick;
  for (int j = 0; j < std::min(kSample, n_levels); ++j) {
    const int l = n_levels == 1 ? 0
                                : (int)std::lround((double)j * (n_levels - 1) / (std::min(kSample, n_levels) - 1));
    if (pick.empty() || pick.back() != l) pick.push_back(l);
  }
  std::vector<double> P, T, n;
  for (int l : pick) {
    P.push_back(pressure[l]);
    T.push_back(temperature[l]);
    n.push_back(density[l]);
  }
  const int L = (int)pick.size();
  const int nsub = marfa_num_subintervals(run->start_wv, run->end_wv);
  CK(ensure(ctx, ctx->b_tune, std::max<size_t>((size_t)L * nsub * NT * 4, 4)), "alloc tuning records");
  const Tune keep = ctx->tune;
  Tune best = keep;
  double best_ms = 1e300;
  // one candidate: the best of two timed calls (the first call also grows buffers)
  auto trial = [&](double &ms) -> int {
    ms = 1e300;
    for (int rep = 0; rep < 3; ++rep) {
      Outputs o;
      o.dev_out = (float *)ctx->b_tune.p;
      int rc = run_levels(ctx, run, L, P.data(), T.data(), n.data(), o, ctx->stream);
      if (!rc) rc = marfa_synchronize(ctx);
      if (rc) return rc;
      double t[8];
      if (rep > 0 && marfa_last_timings(ctx, t) == MARFA_OK) ms = std::min(ms, t[5]);
    }
    return MARFA_OK;
  };
  for (int fcv : {2048, 4096, 8192, 16384})
    for (int ck : {1, 2, 3, 4, 5}) {
      ctx->tune.far_chunk = fcv;
      ctx->tune.coop_k = ck;
      double ms;
      if (int rc = trial(ms)) {
        ctx->tune = keep;
        return rc;
      }
      if (ms < best_ms) {
        best_ms = ms;
        best = ctx->tune;
      }
    }
  // FP32c: the other fine-block shape at the best of the others
  if (run->precision != MARFA_PREC_FP64) {
    ctx->tune = best;
    ctx->tune.fine_pair = !best.fine_pair;
    double ms;
    if (int rc = trial(ms)) {
      ctx->tune = keep;
      return rc;
    }
    if (ms < best_ms) {
      best_ms = ms;
      best = ctx->tune;
    }
  }
  ctx->tune = best;
  if (far_chunk) *far_chunk = best.far_chunk;
  if (coop_k) *coop_k = best.coop_k;
  return MARFA_OK;
}

int marfa_ctx_set_launch(marfa_ctx *ctx, int far_chunk, int coop_k, int fine_pair) {
  if (!ctx) return MARFA_E_ARG;
  if (far_chunk != 2048 && far_chunk != 4096 && far_chunk != 8192 && far_chunk != 16384)
    return set_err(ctx, MARFA_E_ARG, "far_chunk %d (2048, 4096, 8192 or 16384)", far_chunk);
  if (coop_k < 1 || coop_k > 5) return set_err(ctx, MARFA_E_ARG, "coop_k %d (1..5)", coop_k);
  if (fine_pair != 0 && fine_pair != 1) return set_err(ctx, MARFA_E_ARG, "fine_pair %d (0 or 1)", fine_pair);
  ctx->tune.far_chunk = far_chunk;
  ctx->tune.coop_k = coop_k;
  ctx->tune.fine_pair = fine_pair;
  return MARFA_OK;
}

int marfa_ctx_get_launch(marfa_ctx *ctx, int *far_chunk, int *coop_k, int *fine_pair) {
  if (!ctx) return MARFA_E_ARG;
  if (far_chunk) *far_chunk = ctx->tune.far_chunk;
  if (coop_k) *coop_k = ctx->tune.coop_k;
  if (fine_pair) *fine_pair = ctx->tune.fine_pair;
  return MARFA_OK;
}

int marfa_synchronize(marfa_ctx *ctx) {
  if (!ctx) return MARFA_E_ARG;
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "synchronize");
  int herr = 0;
  e = cudaMemcpy(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "d2h err");
  if (herr) return set_err(ctx, herr, "device reported status %d", herr);
  return MARFA_OK;
}

int marfa_eval_count(marfa_ctx *ctx, const marfa_run *run, int n_levels, const double *pressure,
                     const double *temperature, const double *density, int64_t *evals, int64_t *far_evals) {
  if (!ctx) return MARFA_E_ARG;
  if (!evals) return set_err(ctx, MARFA_E_ARG, "evals is null");
  int rc = check_run(ctx, run);
  if (rc) return rc;
  try {
    Plan pl;
    if ((rc = make_plan(ctx, run, pl))) return rc;
    std::vector<LevelConst> lv;
    if ((rc = build_levels(ctx, n_levels, pressure, temperature, density, lv))) return rc;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MARFA_E_CUDA, "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    const int64_t N = ctx->n_lines;
    const int nsub = pl.n_sub, C = (int)pl.chunk_sub.size();
    for (int l = 0; l < n_levels; ++l) {
      evals[l] = 0;
      if (far_evals) far_evals[l] = 0;
    }
    if (C == 0) return MARFA_OK;
    CK(ensure(ctx, ctx->b_nus, (size_t)N * 8), "alloc nus");
    CK(ensure(ctx, ctx->b_gen, (size_t)N * sizeof(LineGen)), "alloc gen");
    CK(ensure(ctx, ctx->b_lv, (size_t)n_levels * sizeof(LevelConst)), "alloc levels");
    CK(ensure(ctx, ctx->b_win, (size_t)nsub * 32), "alloc windows");
    CK(ensure(ctx, ctx->b_chunks, (size_t)C * 20), "alloc chunks");
    CK(ensure(ctx, ctx->b_count, (size_t)C * 16), "alloc count");
    double *d_s = (double *)ctx->b_win.p, *d_e = d_s + nsub;
    int64_t *d_cb = (int64_t *)ctx->b_chunks.p, *d_ce = d_cb + C;
    int *d_cs = (int *)(d_ce + C);
    CK(cudaMemcpyAsync(d_s, pl.s.data(), nsub * 8, cudaMemcpyHostToDevice, st), "h2d");
    CK(cudaMemcpyAsync(d_e, pl.e.data(), nsub * 8, cudaMemcpyHostToDevice, st), "h2d");
    CK(cudaMemcpyAsync(d_cb, pl.chunk_begin.data(), C * 8, cudaMemcpyHostToDevice, st), "h2d");
    CK(cudaMemcpyAsync(d_ce, pl.chunk_end.data(), C * 8, cudaMemcpyHostToDevice, st), "h2d");
    CK(cudaMemcpyAsync(d_cs, pl.chunk_sub.data(), C * 4, cudaMemcpyHostToDevice, st), "h2d");
    CK(cudaMemcpyAsync(ctx->b_lv.p, lv.data(), n_levels * sizeof(LevelConst), cudaMemcpyHostToDevice, st), "h2d");
    CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st), "memset");
    std::vector<unsigned long long> cnt(2 * (size_t)C);
    DeviceLines dl{ctx->d_nu, ctx->d_S, ctx->d_gair, ctx->d_gself, ctx->d_elow, ctx->d_nair, ctx->d_delta, ctx->d_iso, N,
                 ctx->d_S64, ctx->d_gair64};
    for (int l = 0; l < n_levels; ++l) {
      PrepParams pp{};
      pp.lines = dl;
      pp.tips = ctx->d_tips;
      pp.n_iso = ctx->n_iso;
      pp.n_temp = ctx->n_temp;
      pp.tgrid = ctx->tgrid;
      pp.lv = (LevelConst *)ctx->b_lv.p + l;
      pp.n_levels = 1;
      pp.c = make_consts();
      pp.sscale = 1.0;
      pp.nus = (double *)ctx->b_nus.p;
      pp.gen = (LineGen *)ctx->b_gen.p;
      pp.err = ctx->d_err;
      CK(launch_prep(pp, st), "prep kernel");
      CountParams cp;
      cp.nus = pp.nus;
      cp.win = WindowTable{d_s, d_e, nullptr, nullptr, nsub};
      cp.chunk_sub = d_cs;
      cp.chunk_begin = d_cb;
      cp.chunk_end = d_ce;
      cp.n_chunks = C;
      cp.n_levels = 1;
      cp.n_lines = N;
      cp.cutoff = run->cutoff;
      cp.out = (unsigned long long *)ctx->b_count.p;
      CK(launch_count(cp, st), "count kernel");
      CK(cudaMemcpyAsync(cnt.data(), ctx->b_count.p, (size_t)C * 16, cudaMemcpyDeviceToHost, st), "d2h count");
      CK(cudaStreamSynchronize(st), "sync");
      for (int c = 0; c < C; ++c) {
        evals[l] += (int64_t)cnt[2 * (size_t)c];
        if (far_evals) far_evals[l] += (int64_t)cnt[2 * (size_t)c + 1];
      }
    }
    return MARFA_OK;
  } catch (...) {
    return set_err(ctx, MARFA_E_NOMEM, "host allocation failed");
  }
}

int marfa_debug_accumulators(marfa_ctx *ctx, const marfa_run *run, const double *pressure,
                             const double *temperature, const double *density, int n_levels, int level,
                             int isub, double *dump) {
  if (!ctx) return MARFA_E_ARG;
  if (!dump || level < 0 || level >= n_levels || isub < 0 ||
      (run && isub >= marfa_num_subintervals(run->start_wv, run->end_wv)))
    return set_err(ctx, MARFA_E_ARG, "bad dump request");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MARFA_E_CUDA, "cudaSetDevice");
  try {
    std::vector<float> tmp((size_t)n_levels * marfa_num_subintervals(run->start_wv, run->end_wv) * NT);
    Outputs o;
    o.host_out = tmp.data();
    o.host_dump = dump;
    o.dump_level = level;
    o.dump_sub = isub;
    return run_levels(ctx, run, n_levels, pressure, temperature, density, o, ctx->stream);
  } catch (...) {
    return set_err(ctx, MARFA_E_NOMEM, "host allocation failed");
  }
}

int marfa_ctx_set_tips_grid(marfa_ctx *ctx, double t_first, double t_step) {
  if (!ctx) return MARFA_E_ARG;
  if (!std::isfinite(t_first) || !std::isfinite(t_step) || !(t_step > 0.0))
    return set_err(ctx, MARFA_E_ARG, "TIPS grid: bad first temperature %g or step %g", t_first, t_step);
  const TipsGrid g{t_first, t_step};
  int idx = 1;
  double uw = 0.0;
  const double k = (296.0 - t_first) / t_step;
  const bool node = k >= 0.0 && k <= (double)(ctx->n_temp - 1) && (double)(int)k == k;
  if (!node && !tips_node(296.0, g, ctx->n_temp, idx, uw))
    return set_err(ctx, MARFA_E_ARG, "TIPS grid: 296 K outside the table of %d temperatures", ctx->n_temp);
  ctx->tgrid = g;
  ++ctx->alloc_gen; // captured graphs hold the old grid
  return MARFA_OK;
}

int marfa_last_timings(marfa_ctx *ctx, double *times) {
  if (!ctx || !times) return MARFA_E_ARG;
  for (int i = 0; i < 8; ++i) times[i] = 0.0;
  for (auto &m : ctx->marks) {
    float ms = 0.f;
    if (cudaEventSynchronize(m.second.second) != cudaSuccess) return set_err(ctx, MARFA_E_CUDA, "event sync");
    if (cudaEventElapsedTime(&ms, m.second.first, m.second.second) == cudaSuccess) times[m.first] += ms;
  }
  times[6] = ctx->launches;
  times[7] = ctx->far_launches;
  return MARFA_OK;
}

} // extern "C"
