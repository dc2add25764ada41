// marfa_static.cu -- PT record of one level and one subinterval with no
// memory allocation: all device working storage lives in one statically sized
// array of this library.
//
// Who needs this: callers that cannot call cudaMalloc.  Examples are
// applications whose device memory is owned by a pool allocator that
// reserves the whole GPU at start-up and refuses foreign allocations, and
// processes that must not pay cudaMalloc's implicit device synchronisation
// inside a latency-bound loop.  They pass their inputs and output buffer;
// everything else the line-by-line pipeline needs (window line records, per
// line spectroscopy, the shifted-centre order, far-line partial sums, the
// multigrid accumulators and the record itself) is placed in `g_static_scratch`.
//
// The array is `static __device__`: every GPU that loads the library holds
// MARFA_STATIC_SCRATCH_BYTES of it until the process exits.  Host code can
// not use the symbol `g_static_scratch` as a device address (it names a host
// stand-in), so the first call on each device looks up the device address
// with cudaGetSymbolAddress, with that device current, and caches it.  Make
// that first call before any stream capture.  Every call on a device shares
// the array and leaves its contents behind for the next call; calls that
// overlap on the GPU (two host threads, or two streams) race on it.
#include <algorithm>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "marfa_gpu.h"
#include "marfa_kernels.cuh"
#include "marfa_windows.h"

using namespace marfa;

namespace {

constexpr int64_t MAXL = MARFA_STATIC_MAX_WINDOW_LINES;
constexpr int FAR_CHUNK_S = 4096;
constexpr int MAXC = (int)((MAXL + FAR_CHUNK_S - 1) / FAR_CHUNK_S);
constexpr int GSTAGE_LINES = MARFA_STATIC_MAX_NEAR_LINES;

// byte layout of the static array (offsets rounded to 256 B)
constexpr size_t al(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t OFF_NU = 0;
constexpr size_t OFF_F32 = al(OFF_NU + MAXL * 8);            // S, gair, gself, elow, nair, delta
constexpr size_t OFF_ISO = al(OFF_F32 + 6 * MAXL * 4);
constexpr size_t OFF_NUS = al(OFF_ISO + MAXL * 4);
constexpr size_t OFF_GEN = al(OFF_NUS + MAXL * 8);
constexpr size_t OFF_HOT = al(OFF_GEN + MAXL * sizeof(LineGen));
constexpr size_t OFF_RANK = al(OFF_HOT + MAXL * sizeof(Hot64));
constexpr size_t OFF_SNU = al(OFF_RANK + MAXL * 8);
constexpr size_t OFF_SIDX = al(OFF_SNU + MAXL * 8);
constexpr size_t OFF_TIPS = al(OFF_SIDX + MAXL * 4);
constexpr size_t TIPS_MAX = 128 * 1024;                       // doubles of the TIPS table
constexpr size_t OFF_FAR = al(OFF_TIPS + TIPS_MAX * 8);
constexpr size_t OFF_SCR = al(OFF_FAR + (size_t)MAXC * NFAR * 8);
constexpr size_t OFF_GST = al(OFF_SCR + (size_t)SCR_STRIDE * 8);
constexpr size_t OFF_VB = al(OFF_GST + (size_t)GSTAGE_LINES * 52);
constexpr size_t OFF_REC = al(OFF_VB + (size_t)NSLOT * GSTAGE_LINES * 8);
constexpr size_t OFF_SMALL = al(OFF_REC + (size_t)NT * 4);      // tables, level, counters
constexpr size_t SMALL_BYTES = 4096 + (size_t)MAXC * 20;
constexpr size_t TOTAL = al(OFF_SMALL + SMALL_BYTES);
static_assert(TOTAL <= MARFA_STATIC_SCRATCH_BYTES, "static scratch layout exceeds its declared size");

} // namespace

static __device__ __align__(256) unsigned char g_static_scratch[MARFA_STATIC_SCRATCH_BYTES];

namespace {

int fail(char *msg, size_t len, int code, const char *fmt, ...) {
  if (msg && len) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, len, fmt, ap);
    va_end(ap);
  }
  return code;
}

// Device address of g_static_scratch on the current device.  In host code
// the array's name stands for a host-side shadow, not a device address, so
// the address is looked up with the device current -- on every call (a table
// lookup in the runtime once its module is loaded; it allocates nothing), so
// that it stays right after a cudaDeviceReset.
int scratch_address(int dev, unsigned char **out, char *msg, size_t len) {
  if (dev < 0) return fail(msg, len, MARFA_E_ARG, "device index %d out of range", dev);
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess)
    return fail(msg, len, MARFA_E_CUDA, "cudaGetSymbolAddress(static scratch): %s", cudaGetErrorString(e));
  *out = (unsigned char *)p;
  return MARFA_OK;
}

double rec_nu(const marfa_line_record *r, int64_t i) { return *RecordNu{r + i}; }

// The window's packed 36-byte records (copied in one piece) split into the
// field arrays of the kernels, with the isotopologue index jointMolIso / 100
// (LBL.f90:64-65).  Records start 4-byte aligned: every field is read as
// 32-bit words.
__global__ void split_records_kernel(const unsigned *raw, int64_t n, double *nu, float *f32, int *iso, int64_t stride) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned *w = raw + 9 * i; // 36 bytes = 9 words
  nu[i] = __hiloint2double((int)w[1], (int)w[0]);
  for (int f = 0; f < 5; ++f) f32[f * stride + i] = __uint_as_float(w[2 + f]); // S, gair, gself, E, nair
  iso[i] = (int)w[7] / 100;
  f32[5 * stride + i] = __uint_as_float(w[8]); // delta_air
}

cudaError_t split_records(const void *raw, int64_t n, double *nu, float *f32, int *iso, int64_t stride,
                          cudaStream_t st) {
  split_records_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>((const unsigned *)raw, n, nu, f32, iso, stride);
  return cudaGetLastError();
}

} // namespace

extern "C" int marfa_compute_record_static(const marfa_line_record *lines, int64_t n_lines, const double *tips,
                                           int n_iso, int n_temp, const marfa_run *run, double pressure,
                                           double temperature, double density, int isub, float *record,
                                           void *stream, char *msg, size_t msg_len) {
  if (!lines || n_lines < 1 || !tips || n_iso < 1 || n_temp < 139 || !run || !record)
    return fail(msg, msg_len, MARFA_E_ARG, "null or empty argument");
  if ((size_t)n_iso * n_temp > TIPS_MAX)
    return fail(msg, msg_len, MARFA_E_CAPACITY, "TIPS table of %d x %d exceeds %zu values", n_iso, n_temp, TIPS_MAX);
  if (run->target != MARFA_TARGET_ACS && run->target != MARFA_TARGET_VAC) return fail(msg, msg_len, 2, "bad target");
  if (run->chi < 0 || run->chi > 3 || (run->precision != 0 && run->precision != 1) ||
      (run->shape != 0 && run->shape != 1 && run->shape != 100 && run->shape != 101) || !(run->cutoff > 0.0) ||
      run->cutoff > 4000.0)
    return fail(msg, msg_len, MARFA_E_ARG, "bad run parameters");
  if (run->mol_code < 1 || run->mol_code > 12) return fail(msg, msg_len, 8, "unsupported molecule");
  const int nsub = marfa_num_subintervals(run->start_wv, run->end_wv);
  if (isub < 0 || isub >= nsub) return fail(msg, msg_len, MARFA_E_ARG, "subinterval %d outside [0, %d)", isub, nsub);
  // line window of subinterval isub: starting line (main.f90:196-248) and the
  // lblScheme recurrence with capWV (LBL.f90:41-61, main.f90:138-144), by the
  // binary searches of the regular path on the (sorted) records
  const double cut = run->cutoff;
  std::vector<double> ws, we;
  std::vector<int64_t> wl, wh;
  int bad = -1;
  if (plan_windows_of(RecordNu{lines}, n_lines, run->start_wv, isub + 1, cut, ws, we, wl, wh, bad)) {
    if (bad < 0) return fail(msg, msg_len, MARFA_E_DB, "line list ends before start - cutoff");
    return fail(msg, msg_len, MARFA_E_DB, "line list ends inside the window of subinterval %d", bad);
  }
  const double s = ws[isub];
  const int64_t lo = wl[isub], hi = wh[isub];
  // the searches assume sorted centres; the records the window uses (and the
  // one that ends it) are checked
  for (int64_t i = std::max<int64_t>(lo, 1); i <= hi; ++i)
    if (!(rec_nu(lines, i) >= rec_nu(lines, i - 1))) return fail(msg, msg_len, MARFA_E_UNSORTED, "lines not sorted");
  const int64_t m = hi - lo;
  if (m > MAXL)
    return fail(msg, msg_len, MARFA_E_CAPACITY, "window of %lld lines exceeds the static capacity of %lld lines",
                (long long)m, (long long)MAXL);

  // level constants (main.f90:86-96) and the re-ordering window of the sort
  const Consts c = {3.1415926, std::sqrt(std::log(2.0)), 6.626070e-27 * 2.99792458e10 / 1.3806503e-16,
                    std::sqrt(2.0 * 6.02214076e23 * 1.3806503e-16 * std::log(2.0)) / 2.99792458e10,
                    296.0, 1.3806503e-23, 101325.0, std::sqrt(3.1415926), std::sqrt(1.4)};
  LevelConst lv;
  lv.P = pressure;
  lv.T = temperature;
  lv.density = density;
  lv.pself = density * 10.0 * c.bolsi * temperature / c.stdp;
  lv.perrin_b1 = 0.0888 - 0.16 * std::exp(-(0.00410 * temperature));
  lv.perrin_b2 = 0.0526 * std::exp(-(0.00152 * temperature));
  int tidx = 1;
  double tuw = 0.0;
  if (!tips_node(temperature, TipsGrid{20.0, 2.0}, n_temp, tidx, tuw))
    return fail(msg, msg_len, MARFA_E_TEMPERATURE, "temperature outside TIPS");
  if (!std::isfinite(pressure) || pressure < 0.0 || !std::isfinite(density) || lv.pself > pressure * (1.0 + 1e-6))
    return fail(msg, msg_len, 7, "invalid pressure / density");
  double dmin = 1e300, dmax = -1e300, smax = 0.0;
  for (int64_t i = lo; i < hi; ++i) {
    dmin = std::fmin(dmin, (double)lines[i].delta_air);
    dmax = std::fmax(dmax, (double)lines[i].delta_air);
    smax = std::fmax(smax, std::fabs((double)lines[i].S));
  }
  const double margin = m ? std::fabs((dmax - dmin) * pressure) + 1e-7 + 1e-12 * std::fabs(rec_nu(lines, hi)) : 1.0;
  const bool f64 = run->precision == MARFA_PREC_FP64;
  double sscale = 1.0;
  if (!f64) {
    int E = 60 - (int)std::ceil(std::log2(std::fmax(smax, 1e-300) * 3e7));
    E = E < -100 ? -100 : (E > 120 ? 120 : E);
    sscale = std::ldexp(1.0, E);
  }
  const int chi = run->mol_code == 2 ? run->chi : MARFA_CHI_NONE;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(msg, msg_len, MARFA_E_NODEVICE, "no CUDA device");
  unsigned char *base = nullptr;
  int rc = scratch_address(dev, &base, msg, msg_len);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  auto ck = [&](cudaError_t e, const char *where) {
    if (e != cudaSuccess) rc = fail(msg, msg_len, MARFA_E_CUDA, "%s: %s", where, cudaGetErrorString(e));
    return rc == MARFA_OK;
  };

  // inputs: the window's records in one copy (into the per-line parameter
  // region, which the prep kernel writes only after the split), TIPS, tables
  double *d_nu = (double *)(base + OFF_NU);
  float *d_f32 = (float *)(base + OFF_F32);
  int *d_iso = (int *)(base + OFF_ISO);
  static_assert(sizeof(marfa_line_record) == 36 && 36 <= sizeof(LineGen), "record copy fits the parameter region");
  if (m > 0) {
    if (!ck(cudaMemcpyAsync(base + OFF_GEN, lines + lo, (size_t)m * sizeof(marfa_line_record),
                            cudaMemcpyHostToDevice, st), "h2d lines") ||
        !ck(split_records(base + OFF_GEN, m, d_nu, d_f32, d_iso, MAXL, st), "split records"))
      return rc;
  }
  double *d_tips = (double *)(base + OFF_TIPS);
  if (!ck(cudaMemcpyAsync(d_tips, tips, (size_t)n_iso * n_temp * 8, cudaMemcpyHostToDevice, st), "h2d tips"))
    return rc;
  unsigned char *small = base + OFF_SMALL;
  struct Small {
    double sub_s, sub_e;
    int64_t lo, hi;
    int sub_chunk0[2];
    int err;
    int near;
    int queue;
    LevelConst lv;
    double margin;
  };
  Small hs;
  hs.sub_s = s;
  hs.sub_e = s + DELTA_WV;
  hs.lo = 0;
  hs.hi = m;
  const int C = (int)((m + FAR_CHUNK_S - 1) / FAR_CHUNK_S);
  hs.sub_chunk0[0] = 0;
  hs.sub_chunk0[1] = C;
  hs.err = 0;
  hs.near = 0;
  hs.queue = 0;
  hs.lv = lv;
  hs.margin = margin;
  Small *d_small = (Small *)small;
  if (!ck(cudaMemcpyAsync(d_small, &hs, sizeof hs, cudaMemcpyHostToDevice, st), "h2d tables")) return rc;
  int *d_cs = (int *)(small + 1024);
  int64_t *d_cb = (int64_t *)(small + 1024 + al((size_t)MAXC * 4));
  int64_t *d_ce = d_cb + MAXC;
  {
    int cs[MAXC > 0 ? MAXC : 1];
    int64_t cb[MAXC > 0 ? MAXC : 1], ce[MAXC > 0 ? MAXC : 1];
    for (int k = 0; k < C; ++k) {
      cs[k] = 0;
      cb[k] = (int64_t)k * FAR_CHUNK_S;
      ce[k] = std::min<int64_t>(cb[k] + FAR_CHUNK_S, m);
    }
    if (C > 0 && (!ck(cudaMemcpyAsync(d_cs, cs, C * 4, cudaMemcpyHostToDevice, st), "h2d chunks") ||
                  !ck(cudaMemcpyAsync(d_cb, cb, C * 8, cudaMemcpyHostToDevice, st), "h2d chunks") ||
                  !ck(cudaMemcpyAsync(d_ce, ce, C * 8, cudaMemcpyHostToDevice, st), "h2d chunks")))
      return rc;
    // the host arrays above are on the stack: wait for the copies to finish
    if (!ck(cudaStreamSynchronize(st), "sync tables")) return rc;
  }

  WindowTable win{&d_small->sub_s, &d_small->sub_e, &d_small->lo, &d_small->hi, 1};
  DeviceLines dl{d_nu, d_f32, d_f32 + MAXL, d_f32 + 2 * MAXL, d_f32 + 3 * MAXL, d_f32 + 4 * MAXL,
                 d_f32 + 5 * MAXL, d_iso, m};
  PrepParams pp;
  pp.lines = dl;
  pp.tips = d_tips;
  pp.n_iso = n_iso;
  pp.n_temp = n_temp;
  pp.tgrid = TipsGrid{20.0, 2.0};
  pp.lv = &d_small->lv;
  pp.n_levels = 1;
  pp.c = c;
  pp.sscale = sscale;
  pp.nus = (double *)(base + OFF_NUS);
  pp.gen = (LineGen *)(base + OFF_GEN);
  pp.hot32 = f64 ? nullptr : (Hot32 *)(base + OFF_HOT);
  pp.hot64 = f64 ? (Hot64 *)(base + OFF_HOT) : nullptr;
  pp.err = &d_small->err;
  if (m > 0) {
    if (!ck(launch_prep(pp, st), "prep")) return rc;
    SortParams sp;
    sp.nu = d_nu;
    sp.nus = pp.nus;
    sp.margin = &d_small->margin;
    sp.n = m;
    sp.n_levels = 1;
    sp.rank = (int64_t *)(base + OFF_RANK);
    sp.snu = (double *)(base + OFF_SNU);
    sp.sidx = (int *)(base + OFF_SIDX);
    if (!ck(launch_sort(sp, st), "sort")) return rc;
  }
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
  fp.n_levels = 1;
  fp.n_lines = m;
  fp.cutoff = cut;
  fp.sscale = sscale;
  fp.shape = run->shape;
  fp.c = c;
  fp.out = (double *)(base + OFF_FAR);
  if (!ck(launch_far(fp, run->precision, chi, st), "far")) return rc;
  FineParams fn;
  fn.snu = (double *)(base + OFF_SNU);
  fn.sidx = (int *)(base + OFF_SIDX);
  fn.gen = pp.gen;
  fn.lv = pp.lv;
  fn.win = win;
  fn.n_lines = m;
  fn.unit0 = 0;
  fn.n_units = m > 0 ? 1 : 0;
  fn.cutoff = cut;
  fn.sscale = sscale;
  fn.shape = run->shape;
  fn.c = c;
  fn.scratch = base + OFF_SCR;
  fn.err = &d_small->err;
  fn.gstage = base + OFF_GST;
  fn.gstage_cap = 0;
  fn.gstage_bytes = 0;
  int near = 0;
  if (m > 0) {
    if (!ck(launch_near_count(fn, &d_small->near, st), "near count")) return rc;
    if (!ck(cudaMemcpyAsync(&near, &d_small->near, sizeof near, cudaMemcpyDeviceToHost, st), "d2h near") ||
        !ck(cudaStreamSynchronize(st), "sync near"))
      return rc;
  }
  fn.block_threads = fine_block_threads(run->precision, 1 << 30, 0, 0);
  int smem_lines = 0;
  if (!ck(fine_smem_lines(run->precision, chi, fn.block_threads, &smem_lines), "fine shared memory")) return rc;
  const int smem_max = std::min(f64 ? 4096 : 2816, smem_lines);
  fn.smem_cap = std::max(128, std::min(smem_max, (near + 127) / 128 * 128));
  if (near > fn.smem_cap) {
    if (near > GSTAGE_LINES)
      return fail(msg, msg_len, MARFA_E_CAPACITY, "%d lines near the subinterval exceed the static capacity of %d",
                  near, GSTAGE_LINES);
    fn.gstage_cap = (near + 255) / 256 * 256;
    fn.gstage_bytes = fine_smem_bytes(fn.gstage_cap, f64);
  }
  fn.queue = &d_small->queue;
  fn.order = nullptr;
  fn.grid = 1;
  fn.smem_room = fine_smem_bytes(fn.smem_cap, f64);
  fn.coop_k = 5;
  fn.vbuf = base + OFF_VB;
  fn.vbuf_cap = std::max(fn.smem_cap, fn.gstage_cap);
  fn.vbuf_stride = fine_vbuf_elems(fn.vbuf_cap);
  if (m > 0 && !ck(launch_fine(fn, run->precision, chi, st), "fine")) return rc;
  if (m == 0) { // no line in the window: an all-zero scratch slab and zero far sums
    if (!ck(cudaMemsetAsync(base + OFF_SCR, 0, (size_t)SCR_STRIDE * (f64 ? 8 : 4), st), "zero scratch")) return rc;
  }
  CascadeParams cp;
  cp.scratch = base + OFF_SCR;
  cp.far = fp.out;
  cp.fold = nullptr; // one unit: summed from the chunks in the cascade
  cp.sub_chunk0 = d_small->sub_chunk0;
  cp.lv = pp.lv;
  cp.n_chunks = C;
  cp.n_sub = 1;
  cp.unit0 = 0;
  cp.n_units = 1;
  cp.level_out0 = 0;
  cp.inv_sscale = 1.0 / sscale;
  cp.target = run->target;
  cp.out = (float *)(base + OFF_REC);
  cp.out64 = nullptr;
  cp.dump = nullptr;
  cp.dump_unit = -1;
  if (!ck(launch_cascade(cp, run->precision, st), "cascade")) return rc;
  if (!ck(cudaMemcpyAsync(record, base + OFF_REC, (size_t)NT * 4, cudaMemcpyDefault, st), "copy record")) return rc;
  int herr = 0;
  if (!ck(cudaMemcpyAsync(&herr, &d_small->err, sizeof herr, cudaMemcpyDeviceToHost, st), "d2h err") ||
      !ck(cudaStreamSynchronize(st), "sync"))
    return rc;
  if (herr) return fail(msg, msg_len, herr, "device reported status %d", herr);
  if (msg && msg_len) msg[0] = 0;
  return MARFA_OK;
}
