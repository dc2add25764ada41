// marfa_kernels.cu -- the line-by-line kernels for sm_100a.
//
// Pipeline per chunk of atmospheric levels (one stream, no global atomics in
// any accumulation):
//   prep_kernel     per (level, line) spectroscopy in double: shifted centre,
//                   Doppler / Lorentz HWHM, S(T) (Spectroscopy.f90:38-145,
//                   LBL.f90:64-73).
//   rank/scatter    per level, the lines ordered by shifted centre (the
//                   pressure shift re-orders nearby lines) so that every
//                   multigrid cell's contributing lines are one contiguous run.
//   far_kernel      lines at least 1 cm-1 outside the subinterval: 21 grid-0
//                   evaluations each, one thread per line, register sums,
//                   block reduction (leftLBL / rightLBL grid-0 part); line
//                   tiles staged through shared memory by cp.async.
//   far_fold_kernel the far kernel's chunk partials summed per (level,
//                   subinterval, grid-0 position) for the cascade.
//   fine_kernel     lines within 1 cm-1 of / inside the subinterval: every
//                   remaining accumulator (grid 0 near part, grids 1..9, direct
//                   finest points) gathered per accumulator over its
//                   contiguous run of lines (centerLBL and the fine-grid parts
//                   of leftLBL / rightLBL).
//   cascade_kernel  FP64 cascade interpolation per grid-0 cell subtree plus the
//                   PT-record write (Grids.f90:80-139, main.f90:163-168).
#include <cstdio>
#include <type_traits>
#include "marfa_kernels.cuh"
#include "marfa_wiso.h"

namespace marfa {

__constant__ double c_wiso[MARFA_WISO_LEN];

// ---------------------------------------------------------------- prep
__global__ void __launch_bounds__(256) prep_kernel(PrepParams p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int l = blockIdx.y;
  if (i >= p.lines.n) return;
  const LevelConst lv = p.lv[l];
  const Consts c = p.c;
  const int iso = p.lines.iso[i];
  const size_t o = (size_t)l * p.lines.n + i;
  const double nu = p.lines.nu[i];
  if (iso < 1 || iso > MARFA_WISO_LEN || iso > p.n_iso) {
    atomicMax(p.err, 13);
    p.nus[o] = nu;
    return;
  }
  const double T = lv.T, P = lv.P;
  const double M = c_wiso[iso - 1];
  // shiftedLinePosition, dopplerHWHM, lorentzHWHM (Spectroscopy.f90:38-88)
  const double nus = nu + (double)p.lines.delta[i] * P;
  const double alpha = c.doppler * nus * sqrt(T / M);
  const double gair = p.lines.gair64 ? p.lines.gair64[i] : (double)p.lines.gair[i];
  const double gamma = pow(c.tref / T, (double)p.lines.nair[i]) *
                       (gair * (P - lv.pself) + (double)p.lines.gself[i] * lv.pself);
  // TIPSofT (Spectroscopy.f90:91-115): linear interpolation on the table's grid
  int idx = 1;
  double uw = 0.0;
  double S = 0.0;
  if (!tips_node(T, p.tgrid, p.n_temp, idx, uw)) {
    atomicMax(p.err, 11);
  } else {
    const double *row = p.tips + (size_t)(iso - 1) * p.n_temp;
    const double lw = 1.0 - uw;
    const double Q = lw * row[idx - 1] + uw * row[idx];
    const double Qref = tips_ref(row, p.tgrid, p.n_temp);
    if (!isfinite(Q) || !isfinite(Qref)) atomicMax(p.err, 13);
    // intensityOfT (Spectroscopy.f90:118-145), unshifted nu in the emission term
    const double E = (double)p.lines.elow[i];
    const double boltz = exp(-(c.c2 * E / T)) / exp(-(c.c2 * E / c.tref));
    const double emis = (1.0 - exp(-(c.c2 * nu / T))) / (1.0 - exp(-(c.c2 * nu / c.tref)));
    S = (p.lines.S64 ? p.lines.S64[i] : (double)p.lines.S[i]) * (Qref / Q) * boltz * emis;
  }
  LineGen g;
  g.qx = c.sqln2 / alpha;
  g.vy = c.sqln2 * gamma / alpha;
  g.S = S;
  g.alpha = alpha;
  g.gamma = gamma;
  g.lorA = gamma * S / c.pi;
  p.nus[o] = nus;
  p.gen[o] = g;
  if (p.hot32) {
    Hot32 h;
    h.lorA = (float)(g.lorA * p.sscale);
    h.g2 = (float)(gamma * gamma);
    h.qx = g.qx;
    p.hot32[o] = h;
  }
  if (p.hot64) {
    Hot64 h;
    h.lorA = g.lorA;
    h.g2 = gamma * gamma;
    h.qx = g.qx;
    p.hot64[o] = h;
  }
}

// ---------------------------------------------------------------- sort
// Rank of line i among the shifted centres of its level (ties by index).  A
// line can only change places with lines whose unshifted centre lies within
// the level's shift spread, found by binary search on the sorted centres.
__device__ __forceinline__ int64_t lower_bound_d(const double *a, int64_t n, double x) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t m = (lo + hi) >> 1;
    if (a[m] < x) lo = m + 1; else hi = m;
  }
  return lo;
}
__device__ __forceinline__ int64_t upper_bound_d(const double *a, int64_t n, double x) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t m = (lo + hi) >> 1;
    if (a[m] <= x) lo = m + 1; else hi = m;
  }
  return lo;
}

// Lines of the block's re-ordering window that fit in shared memory: the
// block's 256 lines and the lines within the level's margin of them (at the
// densest Venus levels about 1,000).
constexpr int RANK_TILE = 2048;

// The block's lines share one window [w0, w1) of unshifted centres (every
// line's own window lies inside it, as the centres are sorted): when it fits,
// the centres and shifted keys of the window are staged in shared memory once
// and every thread's searches and comparisons run there; otherwise each
// thread searches and scans the global arrays.  Both give the same rank.
__global__ void __launch_bounds__(256) rank_kernel(SortParams p) {
  __shared__ double s_nu[RANK_TILE], s_key[RANK_TILE];
  __shared__ int64_t s_w[2];
  const int64_t i0 = (int64_t)blockIdx.x * blockDim.x, i = i0 + threadIdx.x;
  const int l = blockIdx.y;
  const int64_t i1 = min(i0 + (int64_t)blockDim.x, p.n); // the block's lines [i0, i1)
  const double *key = p.nus + (size_t)l * p.n;
  const double m = p.margin[l];
  if (threadIdx.x == 0) s_w[0] = lower_bound_d(p.nu, p.n, p.nu[i0] - m);
  if (threadIdx.x == 32) s_w[1] = upper_bound_d(p.nu, p.n, p.nu[i1 - 1] + m);
  __syncthreads();
  const int64_t w0 = s_w[0], w1 = s_w[1];
  if (w1 - w0 <= RANK_TILE) {
    const int w = (int)(w1 - w0);
    for (int j = threadIdx.x; j < w; j += blockDim.x) {
      s_nu[j] = p.nu[w0 + j];
      s_key[j] = key[w0 + j];
    }
    __syncthreads();
    if (i >= p.n) return;
    const int t = (int)(i - w0);
    const double nu = s_nu[t], k = s_key[t];
    int a = 0, b = w; // first window entry with centre >= nu - m
    while (a < b) {
      const int c = (a + b) >> 1;
      if (s_nu[c] < nu - m) a = c + 1; else b = c;
    }
    int e = a, f = w; // first entry with centre > nu + m
    while (e < f) {
      const int c = (e + f) >> 1;
      if (s_nu[c] <= nu + m) e = c + 1; else f = c;
    }
    int64_t r = w0 + a;
    for (int j = a; j < e; ++j) {
      const double kj = s_key[j];
      r += (kj < k) || (kj == k && j < t);
    }
    p.rank[(size_t)l * p.n + i] = r;
    return;
  }
  if (i >= p.n) return;
  const double nu = p.nu[i], k = key[i];
  const int64_t jlo = lower_bound_d(p.nu, p.n, nu - m);
  const int64_t jhi = upper_bound_d(p.nu, p.n, nu + m);
  int64_t r = jlo;
  for (int64_t j = jlo; j < jhi; ++j) {
    const double kj = key[j];
    r += (kj < k) || (kj == k && j < i);
  }
  p.rank[(size_t)l * p.n + i] = r;
}

__global__ void __launch_bounds__(256) scatter_kernel(SortParams p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int l = blockIdx.y;
  if (i >= p.n) return;
  const size_t o = (size_t)l * p.n;
  const int64_t r = p.rank[o + i];
  p.snu[o + r] = p.nus[o + i];
  p.sidx[o + r] = (int)i;
}

// ------------------------------------------------------------ block reduce
// Sum of v over the block (warp shuffles, then warp partials in `red` in
// warp order) stored to dst[0 .. N).
template <int N>
__device__ __forceinline__ void block_reduce_store(double (&v)[N], double *dst, double (*red)[N]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double x = v[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if (lane == 0) red[warp][k] = x;
  }
  __syncthreads();
  if (threadIdx.x < N) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[w][threadIdx.x];
    dst[threadIdx.x] = s;
  }
}

// Warp sums of 16 values per lane by a butterfly reduce-scatter: at the step
// of lane bit w a lane keeps one half of its values and receives its partner's
// copy of that half (w + w/2 + ... + 1 = 15 shuffles, then one across the
// half-warps); lane L ends with the warp's sum of value L & 15.  The order of
// the additions is fixed.
__device__ __forceinline__ double warp_scatter16(double (&a)[16]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int w = 8; w >= 1; w >>= 1) {
    const bool up = (lane & w) != 0;
#pragma unroll
    for (int i = 0; i < w; ++i) {
      const double send = up ? a[i] : a[i + w];
      const double keep = up ? a[i + w] : a[i];
      a[i] = keep + __shfl_xor_sync(0xffffffffu, send, w);
    }
  }
  return a[0] + __shfl_xor_sync(0xffffffffu, a[0], 16);
}

// Sum over the block of 31 values per thread, stored to dst[0 .. 31): two
// butterfly halves per warp, then the warp sums in warp order (red: 32 x 32).
template <typename Real>
__device__ __forceinline__ void block_reduce31(const Real (&v)[31], double *dst, double (*red)[32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double a[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) a[i] = (double)v[i];
  double r = warp_scatter16(a);
  if (lane < 16) red[warp][lane] = r;
#pragma unroll
  for (int i = 0; i < 15; ++i) a[i] = (double)v[16 + i];
  a[15] = 0.0;
  r = warp_scatter16(a);
  if (lane < 15) red[warp][16 + lane] = r;
  __syncthreads();
  if (threadIdx.x < 31) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += red[w][threadIdx.x];
    dst[threadIdx.x] = t;
  }
}

// ---------------------------------------------------------------- far lines
// First grid-0 position index k (0..21) whose distance D + k/2 passes the
// chi-factor boundary b (strictly when `strict`), decided in double.
__device__ __forceinline__ int first_k_past(double D, double b, bool strict) {
  int k = (int)ceil(2.0 * (b - D));
  k = k < 0 ? 0 : (k > NFAR ? NFAR : k);
  auto past = [&](int kk) { double d = D + 0.5 * kk; return strict ? (d > b) : (d >= b); };
  while (k > 0 && past(k - 1)) --k;
  while (k < NFAR && !past(k)) ++k;
  return k;
}

template <int CHI>
struct ChiPieces {
  // piece boundaries, strictness, per-piece factor c and exponent rate r
  // (chi = c * 2^(r * d)); piece 0 is chi = 1.
  int nb;
  double b[3];
  bool strict[3];
  float c[4], r[4];
  __device__ ChiPieces(const LevelConst &lv) {
    const float L2E = 1.4426950408889634f;
    c[0] = 1.f; r[0] = 0.f;
    if (CHI == CHI_TONKOV) {
      nb = 3; b[0] = 3.0; b[1] = 150.0; b[2] = 300.0;
      strict[0] = strict[1] = strict[2] = true;
      c[1] = 1.084f; r[1] = -0.027f * L2E;
      c[2] = 0.208f; r[2] = -0.016f * L2E;
      c[3] = 0.025f; r[3] = -0.009f * L2E;
    } else if (CHI == CHI_POLLACK) {
      nb = 2; b[0] = 3.0; b[1] = 10.0; b[2] = 1e300;
      strict[0] = strict[1] = strict[2] = false;
      c[1] = 1.35f; r[1] = -L2E / 10.f;
      c[2] = 0.614f; r[2] = -L2E / 47.f;
      c[3] = 0.f; r[3] = 0.f;
    } else if (CHI == CHI_PERRIN) {
      nb = 3; b[0] = 3.0; b[1] = 30.0; b[2] = 120.0;
      strict[0] = true; strict[1] = strict[2] = false;
      const double b1 = lv.perrin_b1, b2 = lv.perrin_b2, b3 = 0.0232;
      c[1] = (float)exp(3.0 * b1); r[1] = (float)(-b1 * 1.4426950408889634);
      c[2] = (float)exp(-27.0 * b1 + 30.0 * b2); r[2] = (float)(-b2 * 1.4426950408889634);
      c[3] = (float)exp(-27.0 * b1 - 90.0 * b2 + 120.0 * b3); r[3] = (float)(-b3 * 1.4426950408889634);
    } else {
      nb = 0; b[0] = b[1] = b[2] = 1e300;
      strict[0] = strict[1] = strict[2] = true;
      c[1] = c[2] = c[3] = 1.f; r[1] = r[2] = r[3] = 0.f;
    }
  }
};

// Pairs of floats in one 64-bit register for the packed FP32 instructions
// of sm_100 (add/mul/fma .rn.f32x2: two lanes per instruction, each lane
// rounded as the scalar instruction rounds it).
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 x2_pack(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void x2_unpack(f32x2 v, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 x2_add(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 x2_mul(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 x2_fma(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// Grid-0 sums of the far kernel's FP32 form: positions 2j and 2j + 1 in the
// two lanes of acc[j] (j = 0 .. 9), position 20 in a20.
struct FarAcc {
  f32x2 acc[10];
  float a20;
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int j = 0; j < 10; ++j) acc[j] = 0ull;
    a20 = 0.f;
  }
  // v[k] at distance index k of a line left (position k) or right (position 20 - k)
  __device__ __forceinline__ void add(const float (&v)[NFAR], bool left) {
#pragma unroll
    for (int j = 0; j < 10; ++j)
      acc[j] = x2_add(acc[j], left ? x2_pack(v[2 * j], v[2 * j + 1]) : x2_pack(v[20 - 2 * j], v[19 - 2 * j]));
    a20 += left ? v[20] : v[0];
  }
  // Lorentz (times chi = c 2^(r d), one piece) of one line at the 21
  // distances d_k = fl((N 2^-11 + k/2) + f), two distances per instruction:
  // left lines pair k = 2j, 2j + 1 (positions 2j, 2j + 1), right lines pair
  // k = 19 - 2j, 20 - 2j (positions 2j + 1, 2j, stored swapped so that the
  // lanes match).  ce carries cA 2^(r d_k) from pair to pair by 2^(r)
  // (two distance steps of 1/2).  Two consecutive pairs share one reciprocal
  // per lane (Montgomery's batch inversion: 1/a = b / (ab), 1/b = a / (ab)),
  // which halves the MUFU work; the denominators d^2 + gamma^2 are >= 1 and
  // below 2^24 for every cutoff the library accepts, so their products
  // neither overflow nor flush.
  template <bool WITH_CHI>
  __device__ __forceinline__ void lorentz(bool left, float Nf, float ff, float cA, float g2, float r) {
    const f32x2 ff2 = x2_pack(ff, ff), g22 = x2_pack(g2, g2);
    float e0 = 1.f, step = 1.f;
    if (WITH_CHI) {
      step = ex2_approx(0.5f * r);
      e0 = ex2_approx(r * __fadd_rn(Nf, ff));
    }
    const float c0 = cA * e0, c1 = c0 * step;
    const f32x2 step2 = x2_pack(step * step, step * step);
    if (left) {
      f32x2 base = x2_pack(Nf, Nf + 0.5f), ce = x2_pack(c0, c1);
      const f32x2 one = x2_pack(1.f, 1.f);
#pragma unroll
      for (int j = 0; j < 10; j += 2) {
        const f32x2 dA = x2_add(base, ff2);
        const f32x2 denA = x2_fma(dA, dA, g22);
        base = x2_add(base, one);
        const f32x2 dB = x2_add(base, ff2);
        const f32x2 denB = x2_fma(dB, dB, g22);
        base = x2_add(base, one);
        float p0, p1;
        x2_unpack(x2_mul(denA, denB), p0, p1);
        const f32x2 rp = x2_pack(rcp_approx(p0), rcp_approx(p1));
        acc[j] = x2_fma(ce, x2_mul(rp, denB), acc[j]);
        if (WITH_CHI) ce = x2_mul(ce, step2);
        acc[j + 1] = x2_fma(ce, x2_mul(rp, denA), acc[j + 1]);
        if (WITH_CHI) ce = x2_mul(ce, step2);
      }
      float cl, ch;
      x2_unpack(ce, cl, ch);
      const float d = __fadd_rn(Nf + 10.f, ff);
      a20 += cl * rcp_approx(fmaf(d, d, g2));
    } else {
      // k = 0 at position 20, then pairs (k = 2j + 2, 2j + 1) at positions
      // (18 - 2j, 19 - 2j) = acc[9 - j]
      {
        const float d = __fadd_rn(Nf, ff);
        a20 += c0 * rcp_approx(fmaf(d, d, g2));
      }
      f32x2 base = x2_pack(Nf + 1.f, Nf + 0.5f), ce = x2_pack(c1 * step, c1);
      const f32x2 one = x2_pack(1.f, 1.f);
#pragma unroll
      for (int j = 0; j < 10; j += 2) {
        const f32x2 dA = x2_add(base, ff2);
        const f32x2 denA = x2_fma(dA, dA, g22);
        base = x2_add(base, one);
        const f32x2 dB = x2_add(base, ff2);
        const f32x2 denB = x2_fma(dB, dB, g22);
        base = x2_add(base, one);
        float p0, p1;
        x2_unpack(x2_mul(denA, denB), p0, p1);
        const f32x2 rp = x2_pack(rcp_approx(p0), rcp_approx(p1));
        acc[9 - j] = x2_fma(ce, x2_mul(rp, denB), acc[9 - j]);
        if (WITH_CHI) ce = x2_mul(ce, step2);
        acc[8 - j] = x2_fma(ce, x2_mul(rp, denA), acc[8 - j]);
        if (WITH_CHI) ce = x2_mul(ce, step2);
      }
    }
  }
  __device__ __forceinline__ void store(double (&res)[NFAR]) const {
#pragma unroll
    for (int j = 0; j < 10; ++j) {
      float lo, hi;
      x2_unpack(acc[j], lo, hi);
      res[2 * j] = (double)lo;
      res[2 * j + 1] = (double)hi;
    }
    res[20] = (double)a20;
  }
};

// Asynchronous global -> shared copies (cp.async, sm_80+ form; no barrier or
// mbarrier: a thread's cp.async.wait_group completes its own copies).
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

constexpr int FAR_TH = 256;    // threads per far-kernel block
constexpr int FAR_STAGES = 3;  // line tiles in flight per block

// The far kernel's line parameters (shifted centre and the hot record) staged
// through shared memory by cp.async: tile k holds lines begin + 256 k + t, one
// per thread t, in a ring of FAR_STAGES tiles, so the loads of the next two
// tiles are in flight while a thread evaluates its line of this one.  Each
// thread copies and later reads only its own line of a tile, so its own
// wait_group orders the copy before the read, without a barrier.
template <class Hot>
struct FarTiles {
  struct __align__(16) Tile {
    double nu[FAR_TH];
    Hot hot[FAR_TH];
  };
  static_assert(sizeof(Hot) == 16 || sizeof(Hot) == 24, "hot record of 16 or 24 bytes");
  Tile *ring;
  const double *nus;   // this level's shifted centres
  const Hot *hot;      // this level's hot records
  int64_t begin, end;  // the block's lines
  // copies tile k (lines past the end copy nothing) and commits one group
  __device__ __forceinline__ void issue(int k) const {
    const int64_t i = begin + (int64_t)k * FAR_TH + threadIdx.x;
    if (i < end) {
      Tile &t = ring[k % FAR_STAGES];
      cp_async8(&t.nu[threadIdx.x], nus + i);
      if (sizeof(Hot) == 16) {
        cp_async16(&t.hot[threadIdx.x], hot + i);
      } else {
        const double *src = (const double *)(hot + i);
        double *dst = (double *)&t.hot[threadIdx.x];
        cp_async8(dst, src);
        cp_async8(dst + 1, src + 1);
        cp_async8(dst + 2, src + 2);
      }
    }
    cp_async_commit();
  }
  // tile k has arrived (the FAR_STAGES - 1 tiles after it may be in flight)
  __device__ __forceinline__ void wait() const { cp_async_wait<FAR_STAGES - 1>(); }
  __device__ __forceinline__ double nu(int k) const { return ring[k % FAR_STAGES].nu[threadIdx.x]; }
  __device__ __forceinline__ Hot line(int k) const { return ring[k % FAR_STAGES].hot[threadIdx.x]; }
};

template <bool F64, int CHI>
__global__ void __launch_bounds__(FAR_TH, F64 ? 2 : 4) far_kernel(FarParams p) {
  const int item = blockIdx.x;
  const int l = item / p.n_chunks;
  const int ci = item - l * p.n_chunks;
  const int sub = p.chunk_sub[ci];
  const int64_t begin = p.chunk_begin[ci], end = p.chunk_end[ci];
  const double s = p.win.sub_s[sub], se = p.win.sub_e[sub], cut = p.cutoff;
  const LevelConst lv = p.lv[l];
  const size_t lo = (size_t)l * p.n_lines;
  using HotT = typename std::conditional<F64, Hot64, Hot32>::type;
  __shared__ typename FarTiles<HotT>::Tile ring[FAR_STAGES];
  const FarTiles<HotT> tiles{ring, p.nus + lo, (const HotT *)(F64 ? (const void *)p.hot64 : (const void *)p.hot32) + lo,
                             begin, end};
  const int ntile = (int)((end - begin + FAR_TH - 1) / FAR_TH);
#pragma unroll
  for (int k = 0; k < FAR_STAGES - 1; ++k) tiles.issue(k);
  double res[NFAR];
  if constexpr (F64) {
    double acc[NFAR];
#pragma unroll
    for (int k = 0; k < NFAR; ++k) acc[k] = 0.0;
    for (int k = 0; k < ntile; ++k) {
      tiles.issue(k + FAR_STAGES - 1);
      tiles.wait();
      const int64_t i = begin + (int64_t)k * FAR_TH + threadIdx.x;
      double D;
      bool left;
      if (i >= end || !far_line(tiles.nu(k), s, se, cut, D, left)) continue;
      const Hot64 h = tiles.line(k);
      if ((p.shape == 0 && D * h.qx >= 15.0) || p.shape == 1) { // lorentzShape: region 0 at every offset
        // every position in Lorentz region 0: gamma S / (pi (d^2 + gamma^2)) chi(d)
#pragma unroll
        for (int k = 0; k < NFAR; ++k) {
          const double d = D + 0.5 * k;
          double f = h.lorA / fma(d, d, h.g2);
          if (CHI != CHI_NONE) f *= chi_factor_d<CHI>(d, lv);
          if (left) acc[k] += f; else acc[NFAR - 1 - k] += f;
        }
      } else {
        // some position outside region 0 (or a diagnostic shape): general
        // shape per position into a local buffer, then static accumulation
        const LineGen g = p.gen[lo + i];
        double F[NFAR];
#pragma unroll 1
        for (int k = 0; k < NFAR; ++k) {
          const double d = D + 0.5 * k;
          if (p.shape == 100) F[k] = 1.0;
          else if (p.shape == 101) F[k] = d;
          else F[k] = voigt_general<double, CHI>(d, g, lv, p.c, 1.0);
        }
        if (left) {
#pragma unroll
          for (int k = 0; k < NFAR; ++k) acc[k] += F[k];
        } else {
#pragma unroll
          for (int k = 0; k < NFAR; ++k) acc[NFAR - 1 - k] += F[k];
        }
      }
    }
#pragma unroll
    for (int k = 0; k < NFAR; ++k) res[k] = acc[k];
  } else {
    // plain float sums: one thread adds (lines per block) / 256 lines per
    // position (64 at the default 16,384), the block reduction then runs in
    // double
    FarAcc fa;
    fa.init();
    const ChiPieces<CHI> pc(lv);
    for (int k = 0; k < ntile; ++k) {
      tiles.issue(k + FAR_STAGES - 1);
      tiles.wait();
      const int64_t i = begin + (int64_t)k * FAR_TH + threadIdx.x;
      double D;
      bool left;
      if (i >= end || !far_line(tiles.nu(k), s, se, cut, D, left)) continue;
      const Hot32 h = tiles.line(k);
      if ((p.shape == 0 && D * h.qx >= 15.0) || p.shape == 1) { // lorentzShape: region 0 at every offset
        // Exact split of the double distance: D = N*2^-11 + f, so that
        // d_k = (N*2^-11 + k/2) + f is one correctly rounded float.
        const double Nd = floor(D * 2048.0);
        const float Nf = (float)(Nd * (1.0 / 2048.0));
        const float ff = (float)(D - Nd * (1.0 / 2048.0));
        if (CHI == CHI_NONE) {
          fa.lorentz<false>(left, Nf, ff, h.lorA, h.g2, 0.f);
        } else {
          int kb[3];
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            // positions D .. D + 10: a boundary outside that span (with a
            // margin far above the rounding of D) needs no search
            const double bj = pc.b[j];
            kb[j] = j >= pc.nb || D + 10.0 < bj - 1e-6 ? NFAR
                  : (D > bj + 1e-6 ? 0 : first_k_past(D, bj, pc.strict[j]));
          }
          if (kb[0] == 0 && kb[1] == NFAR) {
            // one chi piece over the whole line: chi(d + k/2) = chi(d) *
            // 2^(r/2)^k, one exponential per line and the factor of each
            // next pair of positions by one multiplication (relative error
            // below 1e-6 after the ten steps)
            fa.lorentz<true>(left, Nf, ff, h.lorA * pc.c[1], h.g2, pc.r[1]);
          } else {
            float F[NFAR];
#pragma unroll
            for (int k = 0; k < NFAR; ++k) {
              const float d = __fadd_rn(Nf + 0.5f * k, ff);
              const int pcs = (k >= kb[0]) + (k >= kb[1]) + (k >= kb[2]);
              const float cc = pcs == 0 ? pc.c[0] : (pcs == 1 ? pc.c[1] : (pcs == 2 ? pc.c[2] : pc.c[3]));
              const float rr = pcs == 0 ? pc.r[0] : (pcs == 1 ? pc.r[1] : (pcs == 2 ? pc.r[2] : pc.r[3]));
              F[k] = (h.lorA * cc * rcp_approx(fmaf(d, d, h.g2))) * ex2_approx(rr * d);
            }
            fa.add(F, left);
          }
        }
      } else {
        const LineGen g = p.gen[lo + i];
        float F[NFAR];
#pragma unroll 1
        for (int k = 0; k < NFAR; ++k) {
          const double d = D + 0.5 * k;
          if (p.shape == 100) F[k] = 1.f;
          else if (p.shape == 101) F[k] = (float)d;
          else F[k] = voigt_general<float, CHI>(d, g, lv, p.c, p.sscale);
        }
        fa.add(F, left);
      }
    }
    fa.store(res);
  }
  __shared__ double red[32][NFAR];
  block_reduce_store<NFAR>(res, p.out + ((size_t)l * p.n_chunks + ci) * NFAR, red);
}

// --------------------------------------------------------------- near lines
// First p in [lo, hi) with pred(p), for pred monotone (false ... true),
// searched by galloping from lo.
template <class Pred>
__device__ __forceinline__ int gallop_lb(int lo, int hi, Pred pred) {
  if (lo >= hi || pred(lo)) return lo;
  int base = lo, step = 1;
  while (base + step < hi && !pred(base + step)) {
    base += step;
    step <<= 1;
  }
  int a = base + 1, b = base + step < hi ? base + step : hi;
  while (a < b) {
    const int m = (a + b) >> 1;
    if (pred(m)) b = m; else a = m + 1;
  }
  return a;
}

template <bool F64>
struct Acc;
template <>
struct Acc<true> {
  double v;
  __device__ __forceinline__ void init() { v = 0.0; }
  __device__ __forceinline__ void add(double x) { v += x; }
  __device__ __forceinline__ double value() const { return v; }
};
template <>
struct Acc<false> {
  Kahan k;
  __device__ __forceinline__ void init() { k.init(); }
  __device__ __forceinline__ void add(float x) { k.add(x); }
  __device__ __forceinline__ double value() const { return k.value(); }
};

// The lines of one (level, subinterval) that lie within 1 cm-1 of the
// subinterval or inside it, in shifted-centre order, compacted to those the
// reference schedule lets contribute (inside the line window, within the
// cutoff, centre lines with UU < 10).  Held in shared memory (or, for very
// dense line lists, in a global staging area) as structure of arrays.
constexpr int NBIN9 = 5120; // grid-9 bins over the 10 cm-1 subinterval

template <bool F64>
struct NearStore {
  using Real = typename std::conditional<F64, double, float>::type;
  double *uu;           // fl(nu' - start)
  double *qx, *vy;
  Real *lorA, *g2, *hum;
  int m, c0, c1;        // near-left [0, c0), centre [c0, c1), near-right [c1, m)
  LevelConst lv;
  double sqrt14;

  // F(X) of line q: region 0 (chi-corrected Lorentz) inline, regions 1-4
  // through the out-of-line voigt_core; lorentzShape (qx = -2) and the
  // diagnostic shapes are marked by qx < 0.
  template <int CHI>
  __device__ __forceinline__ Real evalc(int q, double X) const {
    const double ax = fabs(X);
    const double qxv = qx[q];
    if (qxv < 0.0) { // lorentzShape (marked by qx = -2) or a diagnostic shape
      if (qxv > -1.5) return vy[q] < 0.0 ? (Real)1 : (Real)ax;
      const Real axr = (Real)ax;
      const Real lor = fast_div(lorA[q], axr * axr + g2[q]);
      if (CHI == CHI_NONE) return lor;
      if (sizeof(Real) == 8) return lor * (Real)chi_factor_d<CHI>(ax, lv);
      return lor * (Real)chi_factor_f<CHI>(ax, (float)ax, lv);
    }
    if (ax * qxv >= 15.0) {
      const Real axr = (Real)ax;
      const Real lor = fast_div(lorA[q], axr * axr + g2[q]);
      if (CHI == CHI_NONE) return lor;
      if (sizeof(Real) == 8) return lor * (Real)chi_factor_d<CHI>(ax, lv);
      return lor * (Real)chi_factor_f<CHI>(ax, (float)ax, lv);
    }
    return voigt_core<Real, CHI>(X, qxv, vy[q], lorA[q], g2[q], hum[q], lv.perrin_b1, lv.perrin_b2, sqrt14);
  }
  // centre lines: floor(UU * 2^11) and floor(V * 2^11), V = fl(10 - UU); the
  // bin of grid k is the value shifted right by 11 - k
  const short *n11, *nv11;
  // firstU[b] (b = 0 .. NBIN9): first centre line whose grid-9 bin of UU is
  // >= b; firstV[b] (b = 0 .. NBIN9 + 1): first centre line whose grid-9 bin
  // of V is < b (V falls along the sorted lines).  The lines of any run of
  // bins of any grid, in UU or in V, are one index range read off these.
  const unsigned short *firstU, *firstV;
  __device__ __forceinline__ int bin_u(int b) const { return firstU[min(b, NBIN9)]; }
  __device__ __forceinline__ int bin_v(int b) const { return firstV[min(b, NBIN9 + 1)]; }
};


// Grid-0 and RK(1) contributions of one near line: leftLBL grid-0 cells 2..10
// (near-left), centerLBL walks (centre), rightLBL cells 9..1 (near-right).
// Per-lane sums of the grid-0 near part: each lane adds only the few lines
// it owns (a handful), the block reduction then runs in double.
template <bool F64>
struct Lane {
  typename std::conditional<F64, double, float>::type v;
  __device__ __forceinline__ void init() { v = 0; }
  __device__ __forceinline__ void add(decltype(v) x) { v += x; }
  __device__ __forceinline__ double value() const { return (double)v; }
};

template <bool F64, int CHI>
__device__ __forceinline__ void grid0_line(const NearStore<F64> &st, int q, Lane<F64> &aR, Lane<F64> (&aP)[10],
                                           Lane<F64> (&aM)[10], Lane<F64> (&aL)[10]) {
  const double UU = st.uu[q];
  const int cls = q < st.c0 ? 0 : (q < st.c1 ? 1 : 2);
  const double U = UU - DELTA_WV, V = DELTA_WV - UU;
  const int n0 = UU >= 2.0 ? (int)floor(UU) - 1 : 0;
  const int m0 = V >= 2.0 ? (int)floor(V) - 1 : 0;
#pragma unroll
  for (int e = 0; e <= 10; ++e) {
    bool toL = false, toP = false; // L(e) (RK(1) for e = 0) and P(e+1)
    double X = 0.0;
    if (cls == 0) {
      if (e == 0) { toL = true; X = UU; }
      else if (e == 1) { toP = true; X = UU - 1.0; }
      else { toL = true; toP = e <= 9; X = UU - (double)e; }
    } else if (cls == 2) {
      if (e == 0) { toL = toP = true; X = U + 10.0; }
      else if (e <= 8) { toL = toP = true; X = U + (double)(10 - e); }
      else if (e == 9) { toL = true; X = U + 1.0; }
    } else {
      if (e == 0) { toL = true; toP = n0 >= 1; X = UU; }
      else if (e <= n0) { toL = true; toP = e + 1 <= n0; X = UU - (double)e; }
      else if (e >= 10 - m0) { toP = e <= 9; toL = e >= 11 - m0; X = V - (double)(10 - e); }
    }
    if (toL || toP) {
      const auto f = st.template evalc<CHI>(q, X);
      if (toL) {
        if (e == 0) aR.add(f); else aL[e - 1].add(f);
      }
      if (toP && e <= 9) aP[e].add(f);
    }
  }
#pragma unroll
  for (int m = 1; m <= 10; ++m) {
    bool on = false;
    double X = 0.0;
    if (cls == 0) { on = m >= 2; X = (UU - (double)(m - 1)) - 0.5; }
    else if (cls == 2) { on = m <= 9; X = (U + (double)(10 - m)) + 0.5; }
    else if (m <= n0) { on = true; X = (UU - (double)m) + 0.5; }
    else if (m >= 11 - m0) { on = true; X = (V - (double)(11 - m)) + 0.5; }
    if (on) aM[m - 1].add(st.template evalc<CHI>(q, X));
  }
}

// ----------------------------------------------------------- fine grids
// Grids 1..9 and the direct finest points are computed in ten passes (one
// per grid, then the finest points).  Each pass has two halves:
//   line half  one thread per near line evaluates every cell of the pass's
//              grid that the line's walk visits (centerLBL, and the fine
//              parts of leftLBL / rightLBL).  The line's Kuntz coefficients
//              are computed once per pass (regions 2 and 3 only when the
//              pass's smallest offset can reach them).  Values go to a
//              slot buffer (shared memory when it fits, else an L2-resident
//              per-block slice), slot = position of the cell relative to
//              the line.
//   site half  every value the line half wrote has exactly one owner: the
//              cell pair of grid k (or the four finest points of a grid-9
//              cell) it lands on.  One thread (a lane group on the coarse
//              grids) per owner sums the values of the owner's runs of
//              lines, each value once, in line order.
// The line half applies the placement conditions (derived from
// LineGridCalc.f90:7-674) as integer comparisons of the lines' bins: with
// n = floor(UU / H_k) and W an integer, UU >= a H_k <=> n >= a and
// UU < W H_k <=> n < W (likewise for V = fl(10 - UU) and its bin).  The site
// half needs no condition: which slots a line wrote and where they land
// depend only on the parity of its bin (see pair_cells).
// threads per block: 1024 in the FP32 form (64 registers), 512 in FP64
__host__ __device__ constexpr int fine_threads(bool f64) { return f64 ? 512 : 1024; }
// Resident blocks per SM each launch shape is compiled for: 256-thread blocks
// four per SM, 512-thread FP32c blocks two per SM (the paired shape), the
// widest blocks (1024 threads FP32c, 512 FP64) one per SM.  Every shape has
// 64 registers per thread, except the FP64 one with 128.
__host__ __device__ constexpr int fine_min_blocks(bool f64, int th) {
  return th == 256 ? 4 : (!f64 && th == 512 ? 2 : 1);
}
__device__ __forceinline__ int warp_id() { return threadIdx.x >> 5; }

// Line shape of one near line for the fine passes: region 0 inline, Kuntz
// regions 1-3 as one rational form with the line's coefficients selected by
// region, region 4 through voigt_core.
template <bool F64, int CHI>
struct LineEval {
  using Real = typename std::conditional<F64, double, float>::type;
  double qx, vy;
  Real lorA, g2, hum;
  Real A1, B1, A2, B2;                         // region 1 (Shapes.f90:63-70)
  Real A3, B3, C3, D3, A4, B4, C4, D4;         // region 2 (Shapes.f90:72-86)
  Real A5, B5, C5, D5, E5, A6, B6, C6, D6, E6; // region 3 (Shapes.f90:88-113)

  // xlo: a lower bound of |X| over the evaluations that follow.  Regions 2
  // and 3 need VX + VY < 15 (< 5.5 with VX <= 1 or VY >= 0.02), decided on
  // the same double values as the evaluation, so their coefficients are
  // computed only when the smallest VX = xlo * qx can reach them.
  __device__ __forceinline__ void init(const NearStore<F64> &st, int q, double xlo) {
    qx = st.qx[q];
    vy = st.vy[q];
    lorA = st.lorA[q];
    g2 = st.g2[q];
    hum = st.hum[q];
    const Real Y = (Real)(qx < 0.0 ? 0.0 : vy), Y2 = Y * Y;
    A1 = ((Real)0.2820948 + (Real)0.5641896 * Y2) * Y;
    B1 = (Real)0.5641896 * Y;
    A2 = (Real)0.25 + Y2 + Y2 * Y2;
    B2 = Y2 + Y2 - (Real)1.;
    const Real z = (Real)0;
    A3 = B3 = C3 = D3 = A4 = B4 = C4 = D4 = z;
    A5 = B5 = C5 = D5 = E5 = A6 = B6 = C6 = D6 = E6 = z;
    const double vlo = xlo * qx, slo = vlo + vy;
    if (qx >= 0.0 && !(slo < 15.0)) return;
    A3 = Y * horner<Real>(Y2, 0.56419, 3.10304, 4.65456, 1.05786);
    B3 = Y * horner<Real>(Y2, 1.69257, 0.56419, 2.962);
    C3 = Y * ((Real)1.69257 * Y2 - (Real)2.53885);
    D3 = Y * (Real)0.56419;
    A4 = horner<Real>(Y2, 1.0, 6.0, 10.5, 4.5, 0.5625);
    B4 = horner<Real>(Y2, 4.0, 6.0, 9.0, -4.5);
    C4 = (Real)10.5 + (Real)6.0 * (Y2 - (Real)1.0) * Y2;
    D4 = (Real)4.0 * Y2 - (Real)6.0;
    if (qx >= 0.0 && !(slo < 5.5 && (vlo <= 1.0 || vy >= 0.02))) return;
    A5 = horner<Real>(Y, 0.564224, 7.55895, 49.5213, 204.510, 581.746, 1174.8, 1678.33, 1629.76, 973.778,
                      272.102);
    B5 = horner<Real>(Y, 2.25689, 22.6778, 100.705, 247.198, 336.364, 220.843, -2.34403, -60.5644);
    C5 = horner<Real>(Y, 3.38534, 22.6798, 52.8454, 42.5683, 18.546, 4.58029);
    D5 = horner<Real>(Y, 2.25689, 7.56186, 1.66203, -0.128922);
    E5 = horner<Real>(Y, 0.564224, 0.971457E-3);
    A6 = horner<Real>(Y, 1.0, 13.3988, 88.2674, 369.199, 1074.41, 2256.98, 3447.63, 3764.97, 2802.87, 1280.83,
                      272.102);
    B6 = horner<Real>(Y, 5., 53.5952, 266.299, 793.427, 1549.68, 2037.31, 1758.34, 902.306, 211.678);
    C6 = horner<Real>(Y, 10., 80.3928, 269.292, 479.258, 497.302, 308.186, 78.866);
    D6 = horner<Real>(Y, 10., 53.5952, 92.7586, 55.0293, 22.0353);
    E6 = horner<Real>(Y, 5.0, 13.3988, 1.49645);
  }

  // Region 4 (VY < 0.02, 1 < VX, VX + VY < 5.5) as voigt_eval computes it:
  // the Lorentz asymptote beyond VX = 5 (Spectroscopy.f90:232-241), the
  // Doppler core plus the tabulated Lorentz wing beyond sqrt(14)
  // (Spectroscopy.f90:243-261), else the Doppler core.  Inline, so that the
  // passes of the upper levels (where this region is frequent) make no call.
  __device__ __forceinline__ Real region4(double ax, double VXd, const LevelConst &lv, double sqrt14) const {
    const Real axr = (Real)ax;
    const Real VX = (Real)VXd, VXs = VX * VX;
    if (VXd > 5.0) {
      const Real lor = fast_div(lorA, axr * axr + g2);
      Real chi = (Real)1;
      if (CHI != CHI_NONE)
        chi = (sizeof(Real) == 8) ? (Real)chi_factor_d<CHI>(ax, lv) : (Real)chi_factor_f<CHI>(ax, (float)ax, lv);
      return lor * chi * ((Real)1. + (Real)1.5 / VXs);
    }
    const Real dop = hum * exp_neg(VXs);
    if (VXd > sqrt14) {
      int I = (int)(VXd / 0.5 - 1.00001); // 1-based, truncation
      I = I < 1 ? 1 : (I > 8 ? 8 : I);
      // nodes U_i = 1 + i / 2 and weights W_i, i = 0 .. 8
      auto W = [](int i) {
        return i == 0 ? -0.688 : i == 1 ? 0.2667 : i == 2 ? 0.6338 : i == 3 ? 0.4405 : i == 4 ? 0.2529
             : i == 5 ? 0.1601 : i == 6 ? 0.1131 : i == 7 ? 0.0853 : 0.068;
      };
      const double u0 = 1.0 + 0.5 * (double)(I - 1), u1 = 1.0 + 0.5 * (double)I;
      const Real F = (Real)(2. * (W(I - 1) * (u1 - VXd) + W(I) * (VXd - u0)));
      return dop + lorA / (axr * axr) * ((Real)1. + F);
    }
    return dop;
  }

  __device__ __forceinline__ Real operator()(double X, const LevelConst &lv, double sqrt14) const {
    const double ax = fabs(X);
    if (qx < 0.0) { // diagnostic shapes, or lorentzShape (qx = -2; no chi below |X| = 3)
      if (qx > -1.5) return vy < 0.0 ? (Real)1 : (Real)ax;
      const Real axr = (Real)ax;
      return fast_div(lorA, axr * axr + g2);
    }
    const double VXd = ax * qx;
    if (VXd >= 15.0) {
      const Real axr = (Real)ax;
      const Real lor = fast_div(lorA, axr * axr + g2);
      if (CHI == CHI_NONE) return lor;
      if (sizeof(Real) == 8) return lor * (Real)chi_factor_d<CHI>(ax, lv);
      return lor * (Real)chi_factor_f<CHI>(ax, (float)ax, lv);
    }
    // Kuntz regions 1-3 (Shapes.f90:63-113): one branch per region (a warp
    // runs the regions its lanes need; the Horner forms round exactly as the
    // degree-(4, 5) form with the leading coefficients zero would)
    const double sum = VXd + vy;
    const Real VX = (Real)VXd;
    const Real x = VX * VX;
    Real num, den;
    if (sum >= 15.0) {
      num = B1 * x + A1;
      den = (x + B2) * x + A2;
    } else if (sum >= 5.5) {
      num = ((D3 * x + C3) * x + B3) * x + A3;
      den = (((x + D4) * x + C4) * x + B4) * x + A4;
    } else if (VXd <= 1.0 || vy >= 0.02) {
      num = (((E5 * x + D5) * x + C5) * x + B5) * x + A5;
      den = ((((x + E6) * x + D6) * x + C6) * x + B6) * x + A6;
    } else {
      return region4(ax, VXd, lv, sqrt14);
    }
    return fast_div(num, den) * hum;
  }
};

// Exact int -> double for |n| < 2^51 without the conversion unit: the
// integer is added into the mantissa of 1.5 * 2^52 and the bias removed.
__device__ __forceinline__ double i2d(int n) {
  return __longlong_as_double(0x4338000000000000LL + (long long)n) - 6755399441055744.0;
}

// Line half of pass k (1..9: grid k; 10: finest points) for staged line q.
// The offsets X are exact: UU - e H_k is a multiple of the ulp of UU not
// larger than UU, and so are its neighbours e -+ 1 built from it.
template <bool F64, int CHI>
__device__ void line_pass(const NearStore<F64> &st, int q, int k, typename NearStore<F64>::Real *vb, int cap) {
  // Every offset of the line half is below 3 cm-1 in magnitude (at most
  // 4.5 H_k for centre lines, 2 H_{k-1} for near lines, k >= 1), where each
  // chi factor is exactly 1 (ChiFactors.f90: the factors start at |X| = 3):
  // the shape is evaluated without one.
  LineEval<F64, CHI_NONE> ev;
  const double UU = st.uu[q];
  const int cls = q < st.c0 ? 0 : (q < st.c1 ? 1 : 2);
  // value of slot `slot` at offset X (`site`, the edge / mid / finest point
  // the slot stands for, documents the placement: grid k cell e -> e for its
  // edge e and its mid e; finest point i -> i - 2)
  auto put = [&](int slot, int site, double X) {
    (void)site;
    vb[(size_t)slot * cap + q] = ev(X, st.lv, st.sqrt14);
  };
  if (k <= 9) {
    const double hk = h_k(k), hk1 = h_k(k - 1), hn = h_k(k + 1);
    const int ntk = nt_k(k);
    if (cls == 1) {
      // The walk conditions (LineGridCalc.f90:202-331, 343-484) reduce to the
      // parity of the bins: a line of left bin n >= 2 walks edge n-1 (slot 0),
      // edge n-2 (slot 1) and mid n-1 (slot 3), and for odd n also edge n-3
      // (slot 2) and mid n-2 (slot 4); the right walk likewise with its bin
      // nv (slots 5..9).  Equal to the per-cell rules L(e): e >= 1,
      // UU < (2 floor((e+1)/2) + 2) H_k, P(e+1): UU >= (e+2) H_k, ... for
      // every bin of every grid.
      const int n = st.n11[q] >> (11 - k);
      const int nv = st.nv11[q] >> (11 - k);
      if (n < 2 && nv < 2) return;
      ev.init(st, q, hk); // every offset of a centre walk is at least H_k
      if (n >= 2) {
        const double bL = UU - i2d(n - 1) * hk; // X of edge n-1
        put(0, n - 1, bL);
        put(1, n - 2, bL + hk);
        put(3, n - 1, bL + hn);
        if (n & 1) {
          put(2, n - 3, bL + 2.0 * hk);
          put(4, n - 2, (bL + hk) + hn);
        }
      }
      if (nv >= 2) {
        const double V = DELTA_WV - UU;
        const double bV = V - i2d(nv - 1) * hk; // X of the right-walk edge ntk-nv+1
        put(5, ntk - nv + 1, bV);
        put(6, ntk - nv + 2, bV + hk);
        put(8, ntk - nv + 2, bV + hn);
        if (nv & 1) {
          put(7, ntk - nv + 3, bV + 2.0 * hk);
          put(9, ntk - nv + 3, (bV + hk) + hn);
        }
      }
    } else if (cls == 0) {
      if (UU > -hk1) { // D = -UU < H_{k-1}: cells 1 and 2 (leftLBL labels 20-28, 121-129)
        ev.init(st, q, 0.0);
        const bool own = -UU >= hk;
        if (own) put(0, 0, UU);            // e = 0: P(1)
        put(1, 1, UU - hk);                // e = 1: L(1) when own, P(2)
        put(2, 2, UU - hk1);               // e = 2: L(2)
        if (own) put(3, 1, UU - hn);       // M(1)
        put(4, 2, (UU - hk) - hn);         // M(2)
      }
    } else {
      const double U = UU - DELTA_WV;
      if (U < hk1) { // cells ntk and ntk-1 (rightLBL labels 60-69, 131-139)
        ev.init(st, q, 0.0);
        const bool own = U >= hk;
        if (own) put(0, ntk, U);               // e = ntk: L(ntk)
        put(1, ntk - 1, U + hk);               // e = ntk-1: L(ntk-1), P(ntk) when own
        put(2, ntk - 2, U + hk1);              // e = ntk-2: P(ntk-1)
        if (own) put(3, ntk, U + hn);          // M(ntk)
        put(4, ntk - 1, (U + hk) + hn);        // M(ntk-1)
      }
    }
  } else {
    const double H = HSTEP, H9 = h_k(9);
    if (cls == 1) {
      const int ni = st.n11[q], nv9 = st.nv11[q] >> 2;
      const double b0 = UU - i2d(ni) * H; // in [0, H)
      ev.init(st, q, 0.0);
#pragma unroll
      for (int d = 0; d < 7; ++d) { // left fine loop (LineGridCalc.f90:332-339): i = ni+1-d
        const int i = ni + 1 - d;
        if (i >= 2 && i <= NT && ni < 4 * ((i - 2) / 4) + 8) put(d, i - 2, b0 + (double)d * H);
      }
#pragma unroll
      for (int d = 0; d < 8; ++d) { // right fine loop (LineGridCalc.f90:485-490): i = ni+2+d
        const int i = ni + 2 + d;
        if (i >= 2 && i <= NT && nv9 < (NT - i) / 4 + 2) put(7 + d, i - 2, b0 - (double)(1 + d) * H);
      }
    } else if (cls == 0) {
      if (UU > -H9) { // leftLBL label 29: RK(2..5)
        ev.init(st, q, 0.0);
        put(0, 0, UU - H);
        put(1, 1, (UU - H) - H);
        put(2, 2, (UU + H) - H9);
        put(3, 3, UU - H9);
      }
    } else {
      const double U = UU - DELTA_WV;
      if (U < H9) { // rightLBL label 69: RK(NT..NT-3)
        ev.init(st, q, 0.0);
        put(0, NT - 2, U);
        put(1, NT - 3, U + H);
        put(2, NT - 4, (U + H) + H);
        put(3, NT - 5, (U + H9) - H);
      }
    }
  }
}

// ------------------------------------------------------------ site half
// Cell pair p of grid k: cells A = 2p - 1 and B = 2p (p = 1 .. ntk / 2).
// From the walk conditions (LineGridCalc.f90:202-331 left, :343-484 right,
// as line_pass restates them), a centre line of left bin n walks only the
// pair floor(n / 2), and a centre line of right bin nv only the pair
// ntk / 2 + 1 - floor(nv / 2); which slots it wrote and the accumulators they
// land on depend only on the parity of the bin (c = ntk / 2 + 1 - p):
//   left,  n  = 2p     : L_A s0, P_A s1, M_A s3
//   left,  n  = 2p + 1 : L_B s0, P_B s1, M_B s3, L_A s1, P_A s2, M_A s4
//   right, nv = 2c + 1 : P_A s5, L_A s6, M_A s8, P_B s6, L_B s7, M_B s9
//   right, nv = 2c     : P_B s5, L_B s6, M_B s8
// (P(j), L(j): left / right edge of cell j, the edge values L(e) and
// P(e + 1) being one value.)  Near-left lines with D < H_{k-1} reach pair 1,
// near-right lines with U < H_{k-1} pair ntk / 2; `own` is D >= H_k (U >= H_k):
//   near-left : own: P_A s0, L_A s1, M_A s3;  all: P_B s1, L_B s2, M_B s4
//   near-right: own: L_B s0, M_B s3, P_B s1;  all: L_A s1, M_A s4, P_A s2
// Lines sorted by shifted centre have n rising and nv falling, so each of the
// four bin runs is one index range.  G lanes share a pair: they stride over
// the runs, then a fixed-order group reduction; every lane of the warp calls
// this the same number of times, and a group whose p lies past the grid sums
// nothing and stores nothing.
template <bool F64>
__device__ void pair_cells(const NearStore<F64> &st, int k, int p, int G, const typename NearStore<F64>::Real *vb,
                           int cap, typename NearStore<F64>::Real *scr, int lane) {
  using Real = typename NearStore<F64>::Real;
  const int ntk = nt_k(k), np = ntk >> 1, sh = 9 - k;
  const bool valid = p <= np;
  Acc<F64> PA, MA, LA, PB, MB, LB;
  PA.init(); MA.init(); LA.init(); PB.init(); MB.init(); LB.init();
  if (valid) {
    const Real *v0 = vb, *v1 = vb + cap, *v2 = vb + 2 * (size_t)cap, *v3 = vb + 3 * (size_t)cap,
               *v4 = vb + 4 * (size_t)cap;
    const int q0 = st.bin_u((2 * p) << sh), q1 = st.bin_u((2 * p + 1) << sh), q2 = st.bin_u((2 * p + 2) << sh);
    for (int q = q0 + lane; q < q1; q += G) {
      LA.add(v0[q]);
      PA.add(v1[q]);
      MA.add(v3[q]);
    }
    for (int q = q1 + lane; q < q2; q += G) {
      const Real f1 = v1[q];
      LB.add(v0[q]);
      PB.add(f1);
      MB.add(v3[q]);
      LA.add(f1);
      PA.add(v2[q]);
      MA.add(v4[q]);
    }
    const Real *v5 = vb + 5 * (size_t)cap, *v6 = vb + 6 * (size_t)cap, *v7 = vb + 7 * (size_t)cap,
               *v8 = vb + 8 * (size_t)cap, *v9 = vb + 9 * (size_t)cap;
    const int c = np + 1 - p;
    const int r0 = st.bin_v((2 * c + 2) << sh), r1 = st.bin_v((2 * c + 1) << sh), r2 = st.bin_v((2 * c) << sh);
    for (int q = r0 + lane; q < r1; q += G) {
      const Real f6 = v6[q];
      PA.add(v5[q]);
      LA.add(f6);
      MA.add(v8[q]);
      PB.add(f6);
      LB.add(v7[q]);
      MB.add(v9[q]);
    }
    for (int q = r1 + lane; q < r2; q += G) {
      PB.add(v5[q]);
      LB.add(v6[q]);
      MB.add(v8[q]);
    }
    if (p == 1) { // near-left lines with D < H_{k-1}, ascending UU: own (D >= H_k) first
      const double hk = h_k(k), hk1 = h_k(k - 1);
      const int qn = gallop_lb(0, st.c0, [&](int q) { return st.uu[q] > -hk1; });
      for (int q = qn + lane; q < st.c0; q += G) {
        if (-st.uu[q] >= hk) {
          PA.add(v0[q]);
          LA.add(v1[q]);
          MA.add(v3[q]);
        }
        PB.add(v1[q]);
        LB.add(v2[q]);
        MB.add(v4[q]);
      }
    }
    if (p == np) { // near-right lines with U < H_{k-1}, ascending U: own (U >= H_k) last
      const double hk = h_k(k), hk1 = h_k(k - 1);
      const int qn = gallop_lb(st.c1, st.m, [&](int q) { return (st.uu[q] - DELTA_WV) >= hk1; });
      for (int q = st.c1 + lane; q < qn; q += G) {
        if ((st.uu[q] - DELTA_WV) >= hk) {
          LB.add(v0[q]);
          MB.add(v3[q]);
          PB.add(v1[q]);
        }
        LA.add(v1[q]);
        MA.add(v4[q]);
        PA.add(v2[q]);
      }
    }
  }
  double v[6] = {PA.value(), MA.value(), LA.value(), PB.value(), MB.value(), LB.value()};
  for (int off = G >> 1; off > 0; off >>= 1)
#pragma unroll
    for (int i = 0; i < 6; ++i) v[i] += __shfl_down_sync(0xffffffffu, v[i], off, G);
  const double pa = v[0], ma = v[1], la = v[2], pb = v[3], mb = v[4], lb = v[5];
  if (valid && lane == 0) {
    const int a = base_k(k) - NT0 + 2 * p - 2; // cell A; cell B follows
    scr[SCR_FINE_P + a] = (Real)pa;
    scr[SCR_FINE_M + a] = (Real)ma;
    scr[SCR_FINE_L + a] = (Real)la;
    scr[SCR_FINE_P + a + 1] = (Real)pb;
    scr[SCR_FINE_M + a + 1] = (Real)mb;
    scr[SCR_FINE_L + a + 1] = (Real)lb;
  }
}

// Site half of the finest pass for the four points i = 4j-2 .. 4j+1 of
// grid-9 cell j.  They share both outer bounds: the left fine loop ends at
// (4 floor((i-2)/4) + 8) H = (4j + 4) H and the right fine loop's V bound is
// (floor((NT-i)/4) + 2) H9 = (5122 - j) H9, so every line of the run
// [first V < (5122 - j) H9, first UU >= (4j + 4) H) reaches all four points:
// point i through its left loop (slot floor(UU/H) + 1 - i) when
// floor(UU/H) >= i - 1, else through its right loop (slot
// 7 + i - floor(UU/H) - 2).  Then the near lines: RK(2..5) from the
// near-left lines with D < H9, RK(NT-3..NT) from the near-right lines with
// U < H9.
template <bool F64>
__device__ void quad_points(const NearStore<F64> &st, int j, const typename NearStore<F64>::Real *vb, int cap,
                            typename NearStore<F64>::Real *scr) {
  using Real = typename NearStore<F64>::Real;
  const double H9 = h_k(9);
  const int i0 = 4 * j - 2;
  Real *o = scr + SCR_RK + i0 - 2;
  Acc<F64> a[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) a[p].init();
  const int q0 = st.bin_v(5122 - j), q1 = st.bin_u(j + 1);
  for (int q = q0; q < q1; ++q) {
    const int ni = st.n11[q];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int i = i0 + p;
      const int slot = ni >= i - 1 ? ni + 1 - i : 5 + i - ni;
      a[p].add(vb[(size_t)slot * cap + q]);
    }
  }
  if (j == 1) { // RK(2..5): near-left lines with D < H9
    const int qn = gallop_lb(0, st.c0, [&](int q) { return st.uu[q] > -H9; });
    for (int q = qn; q < st.c0; ++q)
#pragma unroll
      for (int p = 0; p < 4; ++p) a[p].add(vb[(size_t)p * cap + q]);
  }
  if (j == NBIN9) { // RK(NT-3..NT): near-right lines with U < H9
    const int qn = gallop_lb(st.c1, st.m, [&](int q) { return (st.uu[q] - DELTA_WV) >= H9; });
    for (int q = st.c1; q < qn; ++q)
#pragma unroll
      for (int p = 0; p < 4; ++p) a[p].add(vb[(size_t)(NT - i0 - p) * cap + q]);
  }
#pragma unroll
  for (int p = 0; p < 4; ++p) o[p] = (Real)a[p].value();
}

__device__ __forceinline__ int block_excl_scan(int v, int &total) {
  __shared__ int ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < nw ? ws[lane] : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += y;
    }
    if (lane < nw) ws[lane] = w;
  }
  __syncthreads();
  total = ws[nw - 1];
  const int r = x - v + (warp > 0 ? ws[warp - 1] : 0);
  __syncthreads();
  return r;
}

// One (level, subinterval) unit: near lines staged, grid 0 reduced, then the
// ten passes of the fine grids.
template <bool F64, int CHI>
__device__ void fine_unit(const FineParams &p, int ub, unsigned char *fine_smem) {
  using Real = typename NearStore<F64>::Real;
  const int u = p.unit0 + ub;
  const int l = u / p.win.n_sub, sub = u - l * p.win.n_sub;
  const double *snu = p.snu + (size_t)l * p.n_lines;
  const int *sidx = p.sidx + (size_t)l * p.n_lines;
  const LineGen *gen = p.gen + (size_t)l * p.n_lines;
  const double s = p.win.sub_s[sub], se = p.win.sub_e[sub], cut = p.cutoff;
  const int64_t wlo = p.win.lo[sub], whi = p.win.hi[sub];
  __shared__ int64_t sb[4];
  // [a, c0): near-left; [c0, c1): centre; [c1, b): near-right (sorted order)
  if (threadIdx.x < 128) { // warp w finds bound w
    const int64_t v = near_bound_warp(snu, p.n_lines, s, se, threadIdx.x >> 5);
    if ((threadIdx.x & 31) == 0) sb[threadIdx.x >> 5] = v;
  }
  __syncthreads();
  const int64_t a = sb[0], b = sb[3];
  const int cnt = (int)(b - a);
  // staging area: shared memory at this unit's own size, or this block's
  // slice of the global staging buffer
  const bool staged_smem = cnt <= p.smem_cap;
  const int cap = staged_smem ? max(32, (cnt + 31) & ~31) : p.gstage_cap;
  unsigned char *base = staged_smem ? fine_smem : (unsigned char *)p.gstage + (size_t)blockIdx.x * p.gstage_bytes;
  NearStore<F64> st;
  st.uu = (double *)base;
  st.qx = st.uu + cap;
  st.vy = st.qx + cap;
  st.lorA = (Real *)(st.vy + cap);
  st.g2 = st.lorA + cap;
  st.hum = st.g2 + cap;
  short *n11 = (short *)(st.hum + cap), *nv11 = n11 + cap;
  st.n11 = n11;
  st.nv11 = nv11;
  st.lv = p.lv[l];
  st.sqrt14 = p.c.sqrt14;
  const double sscale = F64 ? 1.0 : p.sscale;
  // compaction: lines inside the window, within the cutoff, able to contribute
  int m_total = 0, c0 = 0, c1 = 0;
  for (int64_t q0 = a; q0 < b; q0 += blockDim.x) {
    const int64_t q = q0 + threadIdx.x;
    int keep = 0, cls = 1;
    double UU = 0.0;
    int64_t li = 0;
    LineGen g{};
    if (q < b) {
      li = sidx[q];
      keep = near_keep(snu[q], li, s, se, cut, wlo, whi, UU, cls);
      if (keep && p.shape <= 1) g = gen[li]; // in flight during the scan
    }
    int tot;
    const int pos = m_total + block_excl_scan(keep, tot);
    const bool put = keep && pos < cap;
    if (put) {
      st.uu[pos] = UU;
      // bins of the centre lines (UU in [0, 10)): at most 20480
      n11[pos] = cls == 1 ? (short)(int)floor(UU * 2048.0) : (short)0;
      nv11[pos] = cls == 1 ? (short)(int)floor((DELTA_WV - UU) * 2048.0) : (short)0;
      if (p.shape <= 1) {
        const ShapeP<Real> sp = shape_params<Real>(g, p.c, sscale);
        st.qx[pos] = p.shape == 1 ? -2.0 : sp.qx; // -2 marks lorentzShape
        st.vy[pos] = sp.vy;
        st.lorA[pos] = sp.lorA;
        st.g2[pos] = sp.g2;
        st.hum[pos] = sp.hum;
      } else { // diagnostic shapes: F = 1 (vy < 0) or F = |X|
        st.qx[pos] = -1.0;
        st.vy[pos] = p.shape == 100 ? -1.0 : 1.0;
        st.lorA[pos] = st.g2[pos] = st.hum[pos] = (Real)0;
      }
    }
    // staged lines of each class (block-wide counts, one barrier each)
    c0 += __syncthreads_count(put && cls == 0);
    c1 += __syncthreads_count(put && cls != 2);
    m_total += tot;
  }
  st.m = min(m_total, cap);
  st.c0 = c0;
  st.c1 = c1;
  Real *scr = (Real *)p.scratch + (size_t)ub * SCR_STRIDE;
  if (m_total > cap) { // cannot happen when the host sized the staging area
    if (threadIdx.x == 0) atomicMax(p.err, 14);
    __syncthreads();
    return;
  }
  // grid-9 bin tables of the centre lines, built after grid 0; the block
  // reduction of grid 0 uses the same shared memory before them
  __shared__ union {
    struct {
      unsigned short u[NBIN9 + 1], v[NBIN9 + 2];
    } first;
    double red[32][32];
  } s_tab;
  // grid 0 and RK(1): one thread per near line, block reduction
  {
    Lane<F64> aR, aP[10], aM[10], aL[10];
    aR.init();
#pragma unroll
    for (int j = 0; j < 10; ++j) { aP[j].init(); aM[j].init(); aL[j].init(); }
    for (int q = threadIdx.x; q < st.m; q += blockDim.x) grid0_line<F64, CHI>(st, q, aR, aP, aM, aL);
    Real v[31];
    v[0] = aR.v;
#pragma unroll
    for (int j = 0; j < 10; ++j) {
      v[1 + j] = aP[j].v;
      v[11 + j] = aM[j].v;
      v[21 + j] = aL[j].v;
    }
    __shared__ double g0[31];
    block_reduce31<Real>(v, g0, s_tab.red);
    __syncthreads();
    if (threadIdx.x < 31) scr[threadIdx.x] = (Real)g0[threadIdx.x];
  }
  // bins of UU rise and bins of V fall along the sorted lines: firstU[b] for
  // b in (bin(q-1), bin(q)] and firstV[b] for b in (vbin(q), vbin(q-1)] are
  // written by line q, so every entry is written once
  for (int q = st.c0 + threadIdx.x; q <= st.c1; q += blockDim.x) {
    const int bq = q < st.c1 ? min(st.n11[q] >> 2, NBIN9) : NBIN9 + 1;
    const int bp = q > st.c0 ? min(st.n11[q - 1] >> 2, NBIN9) : -1;
    for (int bb = bp + 1; bb <= min(bq, NBIN9); ++bb) s_tab.first.u[bb] = (unsigned short)q;
    const int vq = q < st.c1 ? st.nv11[q] >> 2 : -1;              // <= NBIN9
    const int vp = q > st.c0 ? st.nv11[q - 1] >> 2 : NBIN9 + 1;
    for (int bb = vq + 1; bb <= vp; ++bb) s_tab.first.v[bb] = (unsigned short)q;
  }
  __syncthreads();
  st.firstU = s_tab.first.u;
  st.firstV = s_tab.first.v;

  // slot buffer: in shared memory behind this unit's staged lines when its
  // rows fit in the launch's dynamic shared memory, else this block's global
  // slice
  Real *vb_g = (Real *)p.vbuf + (size_t)blockIdx.x * p.vbuf_stride;
  const size_t stage_bytes = (size_t)cap * (24 + 3 * sizeof(Real) + 4);
  Real *vb_s = (Real *)(fine_smem + stage_bytes);
  for (int k = 1; k <= 10; ++k) {
    const int rows = k <= 9 ? 10 : NSLOT;
    const bool vsm = staged_smem && stage_bytes + (size_t)rows * cap * sizeof(Real) <= p.smem_room;
    Real *vb = vsm ? vb_s : vb_g;
    const int vcap = vsm ? cap : p.vbuf_cap;
    for (int q = threadIdx.x; q < st.m; q += blockDim.x) line_pass<F64, CHI>(st, q, k, vb, vcap);
    __syncthreads();
    if (k <= 9) {
      const int np = nt_k(k) >> 1;
      // lanes per cell pair on grids 1..coop_k: the largest power of two (at
      // most a warp) with which all pairs are summed in one round (about the
      // same number of lines per lane on every grid: the lines per pair halve
      // as the pairs double); one thread per pair on the other grids
      int G = 1;
      if (k <= p.coop_k) {
        const int want = (int)blockDim.x / np;
        G = want >= 32 ? 32 : want >= 16 ? 16 : want >= 8 ? 8 : want >= 4 ? 4 : want >= 2 ? 2 : 1;
      }
      const int lane = threadIdx.x & (G - 1), grp = threadIdx.x / G, ngrp = blockDim.x / G;
      const int rounds = (np + ngrp - 1) / ngrp; // the same for every lane
      for (int r = 0; r < rounds; ++r) pair_cells<F64>(st, k, 1 + grp + r * ngrp, G, vb, vcap, scr, lane);
    } else {
      for (int j = 1 + threadIdx.x; j <= NBIN9; j += blockDim.x) quad_points<F64>(st, j, vb, vcap, scr);
    }
    __syncthreads();
  }
}

// Persistent: every block takes units from the work queue until it is empty
// (units in the given order, most near lines first).
template <bool F64, int CHI, int TH>
__global__ void __launch_bounds__(TH, fine_min_blocks(F64, TH)) fine_kernel(FineParams p) {
  extern __shared__ __align__(16) unsigned char fine_smem[];
  __shared__ int s_unit;
  for (;;) {
    if (threadIdx.x == 0) {
      const int t = atomicAdd(p.queue, 1);
      s_unit = t < p.n_units ? (p.order ? p.order[t] : t) : -1;
    }
    __syncthreads();
    const int ub = s_unit;
    __syncthreads();
    if (ub < 0) break;
    fine_unit<F64, CHI>(p, ub, fine_smem);
  }
}

// Upper bound of the near-line count of every unit (lines with shifted
// centre within 1 cm-1 of, or inside, the subinterval).
__global__ void near_count_kernel(FineParams p, int *counts) {
  const int ub = blockIdx.x * blockDim.x + threadIdx.x;
  if (ub >= p.n_units) return;
  const int u = p.unit0 + ub;
  const int l = u / p.win.n_sub, sub = u - l * p.win.n_sub;
  const double *snu = p.snu + (size_t)l * p.n_lines;
  const double s = p.win.sub_s[sub], se = p.win.sub_e[sub];
  int64_t lo = 0, hi = p.n_lines;
  while (lo < hi) {
    const int64_t m = (lo + hi) >> 1;
    const double v = snu[m];
    if (!(v < s && (v - s) <= -1.0)) hi = m; else lo = m + 1;
  }
  const int64_t a = lo;
  lo = a;
  hi = p.n_lines;
  while (lo < hi) {
    const int64_t m = (lo + hi) >> 1;
    const double v = snu[m];
    if (v > se && ((v - s) - DELTA_WV) >= 1.0) hi = m; else lo = m + 1;
  }
  counts[ub] = (int)(lo - a);
}

// ----------------------------------------------------------------- cascade
// interpolation_step (Grids.f90:80-102): quarter-point value of a coarse
// cell, with the reference's clamp to the half sum.
__device__ __forceinline__ double quarter(double near_edge, double mid, double far_edge) {
  double A = 0.375 * near_edge + 0.75 * mid - 0.125 * far_edge;
  if (A < near_edge || A < mid) A = 0.5 * (near_edge + mid);
  return A;
}

template <bool F64>
__global__ void __launch_bounds__(256) cascade_kernel(CascadeParams p) {
  using Real = typename std::conditional<F64, double, float>::type;
  const int ub = blockIdx.x / NT0;        // unit within the batch
  const int J = blockIdx.x - ub * NT0 + 1; // grid-0 cell of this subtree
  const int u = p.unit0 + ub;
  const int l = u / p.n_sub, sub = u - l * p.n_sub;
  const Real *scr = (const Real *)p.scratch + (size_t)ub * SCR_STRIDE;
  const double inv = p.inv_sscale;
  __shared__ float outb[2048];
  // grid-0 cell J: far-line sums (every warp reduces them itself, in the same
  // order) plus the near part
  double f[4];
  far_sums(p.fold ? p.fold + ((size_t)l * p.n_sub + sub) * NFAR : nullptr,
           p.far + ((size_t)l * p.n_chunks) * NFAR, p.sub_chunk0[sub], p.sub_chunk0[sub + 1], J, f);
  double cP = (f[0] + (double)scr[1 + J - 1]) * inv;
  double cM = (f[1] + (double)scr[11 + J - 1]) * inv;
  double cL = (f[2] + (double)scr[21 + J - 1]) * inv;
  // thread t walks its grid-8 cell's chain of ancestors, grids 1 .. 8, then
  // the cell's two grid-9 children (the ancestors of a warp's cells coincide
  // on the coarse grids: those loads are broadcasts; every address is known
  // up front, so the unrolled walk issues the loads together)
  const int t = threadIdx.x;
  auto refine = [&](int k, int c, double &P, double &M, double &L) {
    const int idx = base_k(k) - NT0 + (J - 1) * (1 << k) + c;
    const double oP = (double)scr[SCR_FINE_P + idx] * inv;
    const double oM = (double)scr[SCR_FINE_M + idx] * inv;
    const double oL = (double)scr[SCR_FINE_L + idx] * inv;
    if ((c & 1) == 0) { // finer cell 2J-1 (Grids.f90:86-93)
      P = oP + cP; M = oM + quarter(cP, cM, cL); L = oL + cM;
    } else {            // finer cell 2J (Grids.f90:94-101)
      P = oP + cM; M = oM + quarter(cL, cM, cP); L = oL + cL;
    }
  };
#pragma unroll
  for (int k = 1; k <= 8; ++k) {
    double P, M, L;
    refine(k, t >> (8 - k), P, M, L);
    cP = P; cM = M; cL = L;
  }
  // grid 9 -> finest points RK(4j-2 .. 4j+1), j = grid-9 cell (Grids.f90:121-138)
  const double dens = p.target == 1 ? p.lv[l].density : 1.0;
  const size_t rec = ((size_t)(p.level_out0 + l) * p.n_sub + sub) * NT;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    double P, M, L;
    refine(9, 2 * t + h, P, M, L);
    const int j = (J - 1) * 512 + 2 * t + h + 1;
    const double v[4] = {quarter(P, M, L), M, quarter(L, M, P), L};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = 4 * j - 2 + q; // RK index, 1-based
      const double x = ((double)scr[SCR_RK + i - 2] * inv + v[q]) * dens;
      outb[8 * t + 4 * h + q] = (float)x;
      if (p.out64) p.out64[rec + i - 1] = x;
    }
  }
  if (J == 1 && t == 0) {
    const double x = (f[3] + (double)scr[0]) * inv * dens;
    p.out[rec] = (float)x;
    if (p.out64) p.out64[rec] = x;
  }
  __syncthreads();
  // coalesced write of RK((J-1)*2048+2 .. J*2048+1), 128-bit stores where aligned
  float *dst = p.out + rec + (size_t)(J - 1) * 2048 + 1;
  const int head = (int)((4 - (((uintptr_t)dst >> 2) & 3)) & 3);
  if ((int)threadIdx.x < head) dst[threadIdx.x] = outb[threadIdx.x];
  const int nvec = (2048 - head) >> 2;
  float4 *dv = (float4 *)(dst + head);
  for (int t2 = threadIdx.x; t2 < nvec; t2 += blockDim.x) {
    const int o = head + 4 * t2;
    dv[t2] = make_float4(outb[o], outb[o + 1], outb[o + 2], outb[o + 3]);
  }
  const int tail0 = head + 4 * nvec;
  if ((int)threadIdx.x < 2048 - tail0) dst[tail0 + threadIdx.x] = outb[tail0 + threadIdx.x];
}

// Far-line sums of every (level, subinterval, grid-0 position) over the
// subinterval's far-kernel chunks, in chunk order (one thread each), so that
// the cascade reads its cells' far sums directly.
__global__ void __launch_bounds__(256) far_fold_kernel(const double *far, const int *sub_chunk0, int n_chunks,
                                                       int n_sub, int n_levels, double *fold) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n_levels * n_sub * NFAR) return;
  const int e = (int)(idx % NFAR);
  const int64_t ls = idx / NFAR;
  const int sub = (int)(ls % n_sub), l = (int)(ls / n_sub);
  const double *fl = far + (size_t)l * n_chunks * NFAR;
  double s = 0.0;
  for (int c = sub_chunk0[sub]; c < sub_chunk0[sub + 1]; ++c) s += fl[(size_t)c * NFAR + e];
  fold[idx] = s;
}

// Raw accumulators of one unit in the oracle's layout (diagnostics).
template <bool F64>
__global__ void dump_kernel(CascadeParams p) {
  using Real = typename std::conditional<F64, double, float>::type;
  const int ub = p.dump_unit - p.unit0;
  const int u = p.dump_unit;
  const int l = u / p.n_sub, sub = u - l * p.n_sub;
  const Real *scr = (const Real *)p.scratch + (size_t)ub * SCR_STRIDE;
  const double inv = p.inv_sscale;
  const double *far = p.far + ((size_t)l * p.n_chunks) * NFAR;
  double *d = p.dump;
  for (int t = threadIdx.x; t < NT + 3 * NCELLS; t += blockDim.x) d[t] = 0.0;
  __syncthreads();
  for (int t = threadIdx.x; t < NFAR + 1; t += blockDim.x) {
    double fs = 0.0;
    if (t < NFAR)
      for (int c = p.sub_chunk0[sub]; c < p.sub_chunk0[sub + 1]; ++c) fs += far[(size_t)c * NFAR + t];
    if (t == 0) d[0] = (fs + (double)scr[0]) * inv;               // RK(1)
    if (t < NFAR && (t & 1) == 0) {                              // integer position e
      const int e = t / 2;
      if (e <= 9) d[NT + e] = (fs + (double)scr[1 + e]) * inv;    // P(e+1)
      if (e >= 1) d[NT + 2 * NCELLS + e - 1] = (fs + (double)scr[21 + e - 1]) * inv; // L(e)
    } else if (t < NFAR) {                                       // mid of cell m
      const int m = (t + 1) / 2;
      d[NT + NCELLS + m - 1] = (fs + (double)scr[11 + m - 1]) * inv;
    }
  }
  for (int t = threadIdx.x; t < NFINE_CELLS; t += blockDim.x) {
    d[NT + NT0 + t] = (double)scr[SCR_FINE_P + t] * inv;
    d[NT + NCELLS + NT0 + t] = (double)scr[SCR_FINE_M + t] * inv;
    d[NT + 2 * NCELLS + NT0 + t] = (double)scr[SCR_FINE_L + t] * inv;
  }
  for (int t = threadIdx.x; t < NT - 1; t += blockDim.x) d[1 + t] = (double)scr[SCR_RK + t] * inv;
}

// ------------------------------------------------------------ eval count
// FSHAPE calls of the reference schedule for one line (LineGridCalc.f90).
__device__ __forceinline__ unsigned count_line(double nu, double s, double se, double cut) {
  const double H = HSTEP;
  if (nu < s) {
    const double D = -(nu - s);
    if (D > cut) return 0;
    if (!(D < 1.0)) return 21;
    for (int k = 1; k <= 9; ++k)
      if (!(D < h_k(k))) return 21 + 2 * k;
    return 41;
  }
  if (nu > se) {
    const double U = (nu - s) - DELTA_WV;
    if (U >= cut) return 0;
    if (!(U < 1.0)) return 21;
    for (int k = 1; k <= 8; ++k)
      if (!(U < h_k(k))) return 21 + 2 * k;
    if (!(U < h_k(9))) return 40;
    return 42;
  }
  const double UU = nu - s;
  if (UU >= DELTA_WV) return 0;
  unsigned n = 2; // F(0) and F(UU)
  // left walk: grid k runs when UU >= 2 H_k; I_k = floor(UU/H_k) - 1
  long long I = 0, cells = 0;
  if (UU >= H) {
    for (int k = 0; k <= 9; ++k) {
      const double hk = h_k(k);
      if (k > 0) I *= 2;
      if (UU >= 2.0 * hk) {
        const long long Ik = (long long)floor(UU / hk) - 1;
        cells += Ik - I;
        I = Ik;
      }
    }
    n += (unsigned)(2 * cells) + (unsigned)((long long)floor(UU / H) - 4 * I);
  }
  const double V = DELTA_WV - UU;
  long long III = 0, rc = 0;
  for (int k = 0; k <= 9; ++k) {
    const double hk = h_k(k);
    if (k > 0) III *= 2;
    if (V >= 2.0 * hk) {
      const long long Ik = (long long)floor(V / hk) - 1;
      rc += Ik - III;
      III = Ik;
    }
  }
  const long long npoint = (long long)floor(UU / H) + 2;
  n += 1 + (unsigned)(2 * rc) + (unsigned)((NT - 4 * III) - npoint + 1);
  return n;
}

__global__ void __launch_bounds__(256) count_kernel(CountParams p) {
  const int item = blockIdx.x;
  const int l = item / p.n_chunks;
  const int ci = item - l * p.n_chunks;
  const int sub = p.chunk_sub[ci];
  const double s = p.win.sub_s[sub], se = p.win.sub_e[sub];
  unsigned long long n = 0, nf = 0;
  for (int64_t i = p.chunk_begin[ci] + threadIdx.x; i < p.chunk_end[ci]; i += blockDim.x) {
    const double nu = p.nus[(size_t)l * p.n_lines + i];
    double D;
    bool left;
    n += count_line(nu, s, se, p.cutoff);
    if (far_line(nu, s, se, p.cutoff, D, left)) nf += NFAR;
  }
  __shared__ unsigned long long red[32][2];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    n += __shfl_down_sync(0xffffffffu, n, off);
    nf += __shfl_down_sync(0xffffffffu, nf, off);
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5][0] = n;
    red[threadIdx.x >> 5][1] = nf;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0, tf = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      t += red[w][0];
      tf += red[w][1];
    }
    p.out[2 * (size_t)item] = t;
    p.out[2 * (size_t)item + 1] = tf;
  }
}

// --------------------------------------------------------------- launchers
// the WISO table lives in constant memory, one copy per device
static bool wiso_loaded[256] = {};

cudaError_t launch_prep(const PrepParams &p, cudaStream_t st) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
  if (!wiso_loaded[dev]) {
    e = cudaMemcpyToSymbol(c_wiso, MARFA_WISO_D, sizeof(MARFA_WISO_D));
    if (e != cudaSuccess) return e;
    wiso_loaded[dev] = true;
  }
  dim3 grid((unsigned)((p.lines.n + 255) / 256), (unsigned)p.n_levels);
  prep_kernel<<<grid, 256, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_sort(const SortParams &p, cudaStream_t st) {
  dim3 grid((unsigned)((p.n + 255) / 256), (unsigned)p.n_levels);
  rank_kernel<<<grid, 256, 0, st>>>(p);
  scatter_kernel<<<grid, 256, 0, st>>>(p);
  return cudaGetLastError();
}

template <bool F64>
static void far_dispatch(const FarParams &p, int chi, unsigned nblk, cudaStream_t st) {
  switch (chi) {
  case CHI_TONKOV: far_kernel<F64, CHI_TONKOV><<<nblk, FAR_TH, 0, st>>>(p); break;
  case CHI_POLLACK: far_kernel<F64, CHI_POLLACK><<<nblk, FAR_TH, 0, st>>>(p); break;
  case CHI_PERRIN: far_kernel<F64, CHI_PERRIN><<<nblk, FAR_TH, 0, st>>>(p); break;
  default: far_kernel<F64, CHI_NONE><<<nblk, FAR_TH, 0, st>>>(p); break;
  }
}

cudaError_t launch_far(const FarParams &p, int precision, int chi, cudaStream_t st) {
  const unsigned nblk = (unsigned)p.n_chunks * (unsigned)p.n_levels;
  if (nblk == 0) return cudaSuccess;
  if (precision == 0) far_dispatch<true>(p, chi, nblk, st);
  else far_dispatch<false>(p, chi, nblk, st);
  return cudaGetLastError();
}

// Block size: fine_threads(F64) threads for dense units (the passes have
// many sites and lines), SMALL_TH for workloads whose units have few near
// lines: those are latency bound per unit, and small blocks put several
// units on every SM.  FP32c dense units can also run on PAIR_TH threads, two
// blocks per SM, so that one block's barrier waits overlap the other's work.
constexpr int SMALL_TH = 256;
constexpr int PAIR_TH = 512;

// Dynamic shared memory one block of a launch shape may take: the opt-in
// limit per block minus the kernel's static arrays, and for the paired shape
// its half of the SM's shared memory (less the static arrays and the
// per-block reservation), rounded down to 1 KB.
template <bool F64, int CHI, int TH>
static cudaError_t fine_block_room(size_t *room) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fine_kernel<F64, CHI, TH>);
  if (e != cudaSuccess) return e;
  int dev = 0, optin = 0, per_sm = 0, reserved = 0;
  if ((e = cudaGetDevice(&dev))) return e;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev))) return e;
  if ((e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev))) return e;
  if ((e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev))) return e;
  size_t r = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
  constexpr int mb = fine_min_blocks(F64, TH);
  if (TH != SMALL_TH && mb > 1) {
    const size_t share = (size_t)per_sm / mb, fixed = fa.sharedSizeBytes + (size_t)reserved;
    r = std::min(r, share > fixed ? (share - fixed) / 1024 * 1024 : (size_t)0);
  }
  *room = r;
  return cudaSuccess;
}

template <bool F64, int CHI, int TH>
static cudaError_t fine_launch_th(const FineParams &p, cudaStream_t st) {
  const size_t smem = p.smem_room;
  cudaError_t e = cudaFuncSetAttribute(fine_kernel<F64, CHI, TH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  fine_kernel<F64, CHI, TH><<<p.grid, TH, smem, st>>>(p);
  return cudaGetLastError();
}

template <bool F64, int CHI>
static cudaError_t fine_launch(const FineParams &p, cudaStream_t st) {
  switch (p.block_threads) {
  case SMALL_TH: return fine_launch_th<F64, CHI, SMALL_TH>(p, st);
  case PAIR_TH: return fine_launch_th<F64, CHI, PAIR_TH>(p, st);
  default: return fine_launch_th<F64, CHI, fine_threads(F64)>(p, st);
  }
}

// Shared-memory plan of the fine kernel: large blocks take the whole room a
// block of their shape may have (fine_block_room) and place each unit's slot
// rows there when they fit; small blocks stage `smem_cap` lines, with slot
// rows when those fit too.  Also the resident blocks of the persistent grid.
template <bool F64, int CHI, int TH>
static cudaError_t fine_occupancy_th(int smem_cap, size_t *smem_room, int *blocks) {
  cudaError_t e;
  int dev = 0, sms = 0;
  if ((e = cudaGetDevice(&dev))) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev))) return e;
  size_t room = 0;
  if ((e = fine_block_room<F64, CHI, TH>(&room))) return e;
  size_t smem = room;
  if (TH == SMALL_TH)
    smem = fine_smem_bytes(smem_cap, F64, fine_smem_bytes(smem_cap, F64, NSLOT) <= room ? NSLOT : 0);
  *smem_room = smem;
  if ((e = cudaFuncSetAttribute(fine_kernel<F64, CHI, TH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
    return e;
  int per_sm = 0;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fine_kernel<F64, CHI, TH>, TH, smem)))
    return e;
  *blocks = (per_sm < 1 ? 1 : per_sm) * sms;
  return cudaSuccess;
}

// Most near lines one block stages in shared memory: the room of a block of
// this shape (fine_block_room) over the bytes per line.
template <bool F64, int CHI, int TH>
static cudaError_t fine_stage_limit_th(int *lines) {
  size_t room = 0;
  const cudaError_t e = fine_block_room<F64, CHI, TH>(&room);
  if (e != cudaSuccess) return e;
  *lines = (int)(room / fine_smem_bytes(1, F64, 0)) / 128 * 128;
  return cudaSuccess;
}

template <bool F64, int CHI>
static cudaError_t fine_stage_limit(int threads, int *lines) {
  switch (threads) {
  case SMALL_TH: return fine_stage_limit_th<F64, CHI, SMALL_TH>(lines);
  case PAIR_TH: return fine_stage_limit_th<F64, CHI, PAIR_TH>(lines);
  default: return fine_stage_limit_th<F64, CHI, fine_threads(F64)>(lines);
  }
}

template <bool F64, int CHI>
static cudaError_t fine_occupancy(int threads, int smem_cap, size_t *room, int *blocks) {
  switch (threads) {
  case SMALL_TH: return fine_occupancy_th<F64, CHI, SMALL_TH>(smem_cap, room, blocks);
  case PAIR_TH: return fine_occupancy_th<F64, CHI, PAIR_TH>(smem_cap, room, blocks);
  default: return fine_occupancy_th<F64, CHI, fine_threads(F64)>(smem_cap, room, blocks);
  }
}

template <bool F64>
static cudaError_t fine_dispatch(const FineParams &p, int chi, cudaStream_t st) {
  switch (chi) {
  case CHI_TONKOV: return fine_launch<F64, CHI_TONKOV>(p, st);
  case CHI_POLLACK: return fine_launch<F64, CHI_POLLACK>(p, st);
  case CHI_PERRIN: return fine_launch<F64, CHI_PERRIN>(p, st);
  default: return fine_launch<F64, CHI_NONE>(p, st);
  }
}

template <bool F64>
static cudaError_t fine_occ_dispatch(int chi, int threads, int smem_cap, size_t *room, int *blocks) {
  switch (chi) {
  case CHI_TONKOV: return fine_occupancy<F64, CHI_TONKOV>(threads, smem_cap, room, blocks);
  case CHI_POLLACK: return fine_occupancy<F64, CHI_POLLACK>(threads, smem_cap, room, blocks);
  case CHI_PERRIN: return fine_occupancy<F64, CHI_PERRIN>(threads, smem_cap, room, blocks);
  default: return fine_occupancy<F64, CHI_NONE>(threads, smem_cap, room, blocks);
  }
}

size_t fine_smem_bytes(int cap, bool f64, int rows) {
  const size_t r = f64 ? 8 : 4;
  return (size_t)cap * (24 + 3 * r + 4 + (size_t)rows * r);
}
size_t fine_vbuf_elems(int cap) { return (size_t)NSLOT * cap; }

int fine_block_threads(int precision, int max_near, int small_below, int pair) {
  if (max_near < small_below) return SMALL_TH;
  return precision != 0 && pair ? PAIR_TH : fine_threads(precision == 0);
}

cudaError_t fine_smem_lines(int precision, int chi, int threads, int *lines) {
  const bool f64 = precision == 0;
  switch (chi) {
  case CHI_TONKOV: return f64 ? fine_stage_limit<true, CHI_TONKOV>(threads, lines) : fine_stage_limit<false, CHI_TONKOV>(threads, lines);
  case CHI_POLLACK: return f64 ? fine_stage_limit<true, CHI_POLLACK>(threads, lines) : fine_stage_limit<false, CHI_POLLACK>(threads, lines);
  case CHI_PERRIN: return f64 ? fine_stage_limit<true, CHI_PERRIN>(threads, lines) : fine_stage_limit<false, CHI_PERRIN>(threads, lines);
  default: return f64 ? fine_stage_limit<true, CHI_NONE>(threads, lines) : fine_stage_limit<false, CHI_NONE>(threads, lines);
  }
}

cudaError_t fine_plan(int precision, int chi, int threads, int smem_cap, size_t *smem_room, int *blocks) {
  return precision == 0 ? fine_occ_dispatch<true>(chi, threads, smem_cap, smem_room, blocks)
                        : fine_occ_dispatch<false>(chi, threads, smem_cap, smem_room, blocks);
}

cudaError_t launch_fine(const FineParams &p, int precision, int chi, cudaStream_t st) {
  if (p.n_units == 0) return cudaSuccess;
  return precision == 0 ? fine_dispatch<true>(p, chi, st) : fine_dispatch<false>(p, chi, st);
}

cudaError_t launch_near_count(const FineParams &p, int *counts, cudaStream_t st) {
  if (p.n_units == 0) return cudaSuccess;
  near_count_kernel<<<(p.n_units + 255) / 256, 256, 0, st>>>(p, counts);
  return cudaGetLastError();
}

cudaError_t launch_far_fold(const double *far, const int *sub_chunk0, int n_chunks, int n_sub, int n_levels,
                            double *fold, cudaStream_t st) {
  const int64_t n = (int64_t)n_levels * n_sub * NFAR;
  if (n == 0) return cudaSuccess;
  far_fold_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(far, sub_chunk0, n_chunks, n_sub, n_levels, fold);
  return cudaGetLastError();
}

cudaError_t launch_cascade(const CascadeParams &p, int precision, cudaStream_t st) {
  if (p.n_units == 0) return cudaSuccess;
  const unsigned nblk = (unsigned)p.n_units * NT0;
  if (precision == 0) cascade_kernel<true><<<nblk, 256, 0, st>>>(p);
  else cascade_kernel<false><<<nblk, 256, 0, st>>>(p);
  if (p.dump && p.dump_unit >= p.unit0 && p.dump_unit < p.unit0 + p.n_units) {
    if (precision == 0) dump_kernel<true><<<1, 256, 0, st>>>(p);
    else dump_kernel<false><<<1, 256, 0, st>>>(p);
  }
  return cudaGetLastError();
}

cudaError_t launch_count(const CountParams &p, cudaStream_t st) {
  const unsigned nblk = (unsigned)p.n_chunks * (unsigned)p.n_levels;
  if (nblk == 0) return cudaSuccess;
  count_kernel<<<nblk, 256, 0, st>>>(p);
  return cudaGetLastError();
}

} // namespace marfa
