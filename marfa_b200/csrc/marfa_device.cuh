// marfa_device.cuh -- device-side definitions shared by the line-by-line kernels.
//
// Geometry of the ten-grid multigrid (Grids.f90:6-16, 48-58): grid k (k = 0..9)
// has NT_k = 10 * 2^k cells of width H_k = 2^-k cm-1 over one 10 cm-1
// subinterval; every cell holds a left-edge (P), mid (M) and right-edge (L)
// accumulator; the finest grid has NT = 20481 points with step H = H9 / 4.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace marfa {

constexpr int NT0 = 10;
constexpr int NT = 20481;
constexpr int NCELLS = 10230;             // cells of grids 0..9
constexpr int NFINE_CELLS = NCELLS - NT0; // cells of grids 1..9
constexpr double HSTEP = 0.00048828125;   // H
constexpr double DELTA_WV = 10.0;

__host__ __device__ constexpr int nt_k(int k) { return NT0 << k; }
__host__ __device__ constexpr int base_k(int k) { return NT0 * ((1 << k) - 1); }
// H_k = 2^-k, built from the exponent bits (exact, no library call)
__host__ __device__ inline double h_k(int k) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)(1023 - k) << 52);
#else
  return ldexp(1.0, -k);
#endif
}

// Accumulators of one (level, subinterval) produced by the near-line kernel:
//   [0]            RK(1)
//   [1 .. 10]      P(1..10) of grid 0      [11 .. 20] M      [21 .. 30] L
//   [31 ..)        P, M, L blocks of grids 1..9 (NFINE_CELLS each); cell j of
//                  grid k at base_k(k) - 10 + j - 1
//   [31 + 3*NFINE_CELLS ..)  RK(2..NT) direct finest-grid contributions
constexpr int SCR_G0 = 0;
constexpr int SCR_FINE_P = 31;
constexpr int SCR_FINE_M = SCR_FINE_P + NFINE_CELLS;
constexpr int SCR_FINE_L = SCR_FINE_M + NFINE_CELLS;
constexpr int SCR_RK = SCR_FINE_L + NFINE_CELLS;
constexpr int SCR_LEN = SCR_RK + (NT - 1);
constexpr int SCR_STRIDE = 51200; // >= SCR_LEN, multiple of 64

// Far-line kernel output: sums at the 21 grid-0 positions 0, 0.5, ..., 10
// (index 2 * position) over the lines that are at least 1 cm-1 outside the
// subinterval; each integer position feeds L(e) and P(e+1) of grid 0.
constexpr int NFAR = 21;

// Physical constants of the all-double type map (values from Constants.f90,
// evaluated in double on the host).
struct Consts {
  double pi, sqln2, c2, doppler, tref, bolsi, stdp, sqrtpi, sqrt14;
};

// Per-(level, line) parameters in line-index order.
struct LineGen {     // every field in double
  double qx;         // sqln2 / alpha_D  (VX = |X| * qx)
  double vy;         // sqln2 * gamma_L / alpha_D
  double S;          // intensity at the level temperature
  double alpha;      // Doppler HWHM
  double gamma;      // Lorentz HWHM
  double lorA;       // gamma * S / PI
};
struct Hot32 {       // far-line fast path, FP32-compensated form
  float lorA;        // gamma * S / PI * 2^scale_exp
  float g2;          // gamma^2
  double qx;
};
struct Hot64 {
  double lorA, g2, qx;
};

// Per-level constants.
struct LevelConst {
  double P, T, density, pself;
  double perrin_b1, perrin_b2; // perrin chi-factor temperature terms
};

// ------------------------------------------------------------------- TIPS
// Temperature grid of the partition-sum table: node j (0-based) at
// t0 + j dt.  The reference's table (TIPS(74, 501), Gamache 2017) has
// t0 = 20 K, dt = 2 K; Gamache's 2021 tables use 1 K steps.
struct TipsGrid {
  double t0, dt;
};

// TIPSofT (Spectroscopy.f90:91-115): the lower node index idx (1-based, the
// reference's `int((T - 20) / 2 + 1)`) and the weight uw of node idx + 1 for
// linear interpolation, Q = (1 - uw) row[idx - 1] + uw row[idx]; false when T
// lies outside the table.  On the reference's grid these are its operations.
__host__ __device__ inline bool tips_node(double T, TipsGrid g, int n_temp, int &idx, double &uw) {
  const double tval = (T - g.t0) / g.dt + 1.0;
  if (!(tval >= 1.0) || !(tval < (double)n_temp)) return false; // idx + 1 <= n_temp
  idx = (int)tval;
  const double lwt = (double)(idx - 1) * g.dt + g.t0;
  uw = (T - lwt) / g.dt;
  return true;
}

// Q(296 K) of one row: the node itself when 296 K is a node (node 139 of the
// reference's table, Spectroscopy.f90:136), else the interpolation there.
__host__ __device__ inline double tips_ref(const double *row, TipsGrid g, int n_temp) {
  const double k = (296.0 - g.t0) / g.dt;
  const int ki = (int)k;
  if ((double)ki == k) return row[ki];
  int idx = 1;
  double uw = 0.0;
  tips_node(296.0, g, n_temp, idx, uw);
  return (1.0 - uw) * row[idx - 1] + uw * row[idx];
}

// ---------------------------------------------------------------- Kahan sum
struct Kahan {
  float s, c;
  __device__ __forceinline__ void init() { s = 0.f; c = 0.f; }
  __device__ __forceinline__ void add(float x) {
    float y = __fsub_rn(x, c);
    float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// --------------------------------------------------------------- chi-factors
// ChiFactors.f90:29-122; `ax` = |X| in double decides the piece in both
// precisions, the factor itself is evaluated in the kernel's precision.
enum { CHI_NONE = 0, CHI_TONKOV = 1, CHI_POLLACK = 2, CHI_PERRIN = 3 };

template <int CHI>
__device__ __forceinline__ double chi_factor_d(double ax, const LevelConst &lv) {
  if (CHI == CHI_TONKOV) {
    if (ax > 3.0) {
      if (ax <= 150.0) return 1.084 * exp(-(0.027 * ax));
      if (ax <= 300.0) return 0.208 * exp(-(0.016 * ax));
      return 0.025 * exp(-(0.009 * ax));
    }
    return 1.0;
  } else if (CHI == CHI_POLLACK) {
    if (ax >= 3.0) {
      if (ax < 10.0) return 1.35 * exp(-ax / 10.0);
      return 0.614 * exp(-ax / 47.0);
    }
    return 1.0;
  } else if (CHI == CHI_PERRIN) {
    const double b1 = lv.perrin_b1, b2 = lv.perrin_b2, b3 = 0.0232;
    if (ax > 3.0) {
      if (ax < 30.0) return exp(-(b1 * (ax - 3.0)));
      if (ax < 120.0) return exp(-(b1 * (30.0 - 3.0)) - b2 * (ax - 30.0));
      return exp(-(b1 * (30.0 - 3.0)) - b2 * (120.0 - 30.0) - b3 * (ax - 120.0));
    }
    return 1.0;
  }
  return 1.0;
}

// Same piece decision (made on the double |X|), factor in float.
template <int CHI>
__device__ __forceinline__ float chi_factor_f(double ax, float axf, const LevelConst &lv) {
  const float L2E = 1.4426950408889634f;
  if (CHI == CHI_TONKOV) {
    if (ax > 3.0) {
      if (ax <= 150.0) return 1.084f * ex2_approx(-0.027f * L2E * axf);
      if (ax <= 300.0) return 0.208f * ex2_approx(-0.016f * L2E * axf);
      return 0.025f * ex2_approx(-0.009f * L2E * axf);
    }
    return 1.f;
  } else if (CHI == CHI_POLLACK) {
    if (ax >= 3.0) {
      if (ax < 10.0) return 1.35f * ex2_approx(-(L2E / 10.f) * axf);
      return 0.614f * ex2_approx(-(L2E / 47.f) * axf);
    }
    return 1.f;
  } else if (CHI == CHI_PERRIN) {
    return (float)chi_factor_d<CHI_PERRIN>(ax, lv);
  }
  return 1.f;
}

// Horner evaluation c0*x^n + ... + cn in the order (((c0 x + c1) x + c2) ...),
// the order the Kuntz coefficient polynomials are written in Shapes.f90.
template <typename Real>
__device__ __forceinline__ Real horner_acc(Real acc, Real) { return acc; }
template <typename Real, typename... Rest>
__device__ __forceinline__ Real horner_acc(Real acc, Real x, double c, Rest... rest) {
  return horner_acc<Real>(acc * x + (Real)c, x, rest...);
}
template <typename Real, typename... Rest>
__device__ __forceinline__ Real horner(Real x, double c0, Rest... rest) {
  return horner_acc<Real>((Real)c0, x, rest...);
}

// ------------------------------------------------------- general line shape
// Per-line parameters of the general shape evaluation.  Region decisions use
// qx and vy in double in both precisions; values are computed in Real.
template <typename Real>
struct ShapeP {
  double qx;   // sqln2 / alpha_D
  double vy;   // sqln2 * gamma_L / alpha_D
  Real lorA;   // gamma S / PI (scaled)
  Real g2;     // gamma^2
  Real hum;    // S sqln2 / (sqrt(PI) alpha_D) (scaled)
};

template <typename Real>
__device__ __forceinline__ ShapeP<Real> shape_params(const LineGen &g, const Consts &c, double sscale) {
  ShapeP<Real> s;
  s.qx = g.qx;
  s.vy = g.vy;
  s.lorA = (Real)(g.lorA * sscale);
  s.g2 = (Real)(g.gamma * g.gamma);
  s.hum = (Real)(g.S * sscale * (c.sqln2 / (c.sqrtpi * g.alpha)));
  return s;
}

__device__ __forceinline__ float fast_div(float a, float b) { return a * rcp_approx(b); }
__device__ __forceinline__ double fast_div(double a, double b) { return a / b; }
__device__ __forceinline__ float exp_neg(float x) { return ex2_approx(-x * 1.4426950408889634f); }
__device__ __forceinline__ double exp_neg(double x) { return exp(-x); }

// Humlicek-Kuntz voigt of Shapes.f90:22-133 with the reference's region 0
// and region-4 asymptotics (Spectroscopy.f90:232-261), times the intensity.
// Region chosen from VX = |X| qx and VY in double; formula in Real.
//   region 0 / asym1: chi-corrected Lorentz  lorA / (X^2 + gamma^2) * chi
//   regions 1-3     : Kuntz rational function of VX^2 * hum
//   asym2           : doppler + gamma S / (PI X^2) (1 + F)
//   doppler         : hum * exp(-VX^2)
template <typename Real, int CHI>
__device__ Real voigt_eval(double Xd, const ShapeP<Real> &p, const LevelConst &lv, double sqrt14) {
  const double ax = fabs(Xd);
  const double VXd = ax * p.qx;
  const double VYd = p.vy;
  const Real axr = (Real)ax;
  if (VXd >= 15.0) { // region 0
    const Real lor = fast_div(p.lorA, axr * axr + p.g2);
    if (CHI == CHI_NONE) return lor;
    if (sizeof(Real) == 8) return lor * (Real)chi_factor_d<CHI>(ax, lv);
    return lor * (Real)chi_factor_f<CHI>(ax, (float)ax, lv);
  }
  const Real VX = (Real)VXd, VY = (Real)VYd;
  const Real VXs = VX * VX;
  const double sum = VXd + VYd;
  if (sum >= 15.0) { // region 1
    const Real Y = VY, Y2 = Y * Y;
    const Real A1 = ((Real)0.2820948 + (Real)0.5641896 * Y2) * Y;
    const Real B1 = (Real)0.5641896 * Y;
    const Real A2 = (Real)0.25 + Y2 + Y2 * Y2;
    const Real B2 = Y2 + Y2 - (Real)1.;
    return (A1 + B1 * VXs) / (A2 + B2 * VXs + VXs * VXs) * p.hum;
  }
  if (sum >= 5.5) { // region 2
    const Real Y = VY, Y2 = Y * Y;
    const Real A3 = Y * horner<Real>(Y2, 0.56419, 3.10304, 4.65456, 1.05786);
    const Real B3 = Y * horner<Real>(Y2, 1.69257, 0.56419, 2.962);
    const Real C3 = Y * ((Real)1.69257 * Y2 - (Real)2.53885);
    const Real D3 = Y * (Real)0.56419;
    const Real A4 = horner<Real>(Y2, 1.0, 6.0, 10.5, 4.5, 0.5625);
    const Real B4 = horner<Real>(Y2, 4.0, 6.0, 9.0, -4.5);
    const Real C4 = (Real)10.5 + (Real)6.0 * (Y2 - (Real)1.0) * Y2;
    const Real D4 = (Real)4.0 * Y2 - (Real)6.0;
    return (((D3 * VXs + C3) * VXs + B3) * VXs + A3) /
           ((((VXs + D4) * VXs + C4) * VXs + B4) * VXs + A4) * p.hum;
  }
  if (VXd <= 1.0 || VYd >= 0.02) { // region 3
    const Real Y = VY;
    const Real A5 = horner<Real>(Y, 0.564224, 7.55895, 49.5213, 204.510, 581.746, 1174.8, 1678.33,
                                 1629.76, 973.778, 272.102);
    const Real B5 = horner<Real>(Y, 2.25689, 22.6778, 100.705, 247.198, 336.364, 220.843, -2.34403,
                                 -60.5644);
    const Real C5 = horner<Real>(Y, 3.38534, 22.6798, 52.8454, 42.5683, 18.546, 4.58029);
    const Real D5 = horner<Real>(Y, 2.25689, 7.56186, 1.66203, -0.128922);
    const Real E5 = horner<Real>(Y, 0.564224, 0.971457E-3);
    const Real A6 = horner<Real>(Y, 1.0, 13.3988, 88.2674, 369.199, 1074.41, 2256.98, 3447.63, 3764.97,
                                 2802.87, 1280.83, 272.102);
    const Real B6 = horner<Real>(Y, 5., 53.5952, 266.299, 793.427, 1549.68, 2037.31, 1758.34, 902.306,
                                 211.678);
    const Real C6 = horner<Real>(Y, 10., 80.3928, 269.292, 479.258, 497.302, 308.186, 78.866);
    const Real D6 = horner<Real>(Y, 10., 53.5952, 92.7586, 55.0293, 22.0353);
    const Real E6 = horner<Real>(Y, 5.0, 13.3988, 1.49645);
    return ((((E5 * VXs + D5) * VXs + C5) * VXs + B5) * VXs + A5) /
           (((((VXs + E6) * VXs + D6) * VXs + C6) * VXs + B6) * VXs + A6) * p.hum;
  }
  // region 4
  if (VXd > 5.0) { // voigtAsymptotic1
    const Real lor = fast_div(p.lorA, axr * axr + p.g2);
    Real chi = (Real)1;
    if (CHI != CHI_NONE)
      chi = (sizeof(Real) == 8) ? (Real)chi_factor_d<CHI>(ax, lv) : (Real)chi_factor_f<CHI>(ax, (float)ax, lv);
    return lor * chi * ((Real)1. + (Real)1.5 / VXs);
  }
  const Real dop = p.hum * exp_neg(VXs);
  if (VXd > sqrt14) { // voigtAsymptotic2
    const double Ut[9] = {1., 1.5, 2., 2.5, 3., 3.5, 4., 4.5, 5.};
    const double Wt[9] = {-0.688, 0.2667, 0.6338, 0.4405, 0.2529, 0.1601, 0.1131, 0.0853, 0.068};
    int I = (int)(VXd / 0.5 - 1.00001); // 1-based, truncation
    I = I < 1 ? 1 : (I > 8 ? 8 : I);
    const Real F = (Real)(2. * (Wt[I - 1] * (Ut[I] - VXd) + Wt[I] * (VXd - Ut[I - 1])));
    return dop + p.lorA / (axr * axr) * ((Real)1. + F);
  }
  return dop;
}

// Regions 1-4 only (VX < 15), out of line so that kernels keep one copy of
// the Kuntz polynomials; region 0 is evaluated inline by the callers.
template <typename Real, int CHI>
__device__ __noinline__ Real voigt_core(double Xd, double qx, double vy, Real lorA, Real g2, Real hum,
                                        double pb1, double pb2, double sqrt14) {
  ShapeP<Real> sp;
  sp.qx = qx;
  sp.vy = vy;
  sp.lorA = lorA;
  sp.g2 = g2;
  sp.hum = hum;
  LevelConst lv;
  lv.perrin_b1 = pb1;
  lv.perrin_b2 = pb2;
  return voigt_eval<Real, CHI>(Xd, sp, lv, sqrt14);
}

template <typename Real, int CHI>
__device__ __forceinline__ Real voigt_general(double Xd, const LineGen &g, const LevelConst &lv,
                                              const Consts &c, double sscale) {
  const ShapeP<Real> sp = shape_params<Real>(g, c, sscale);
  const double ax = fabs(Xd);
  if (ax * sp.qx >= 15.0) { // region 0 inline
    const Real axr = (Real)ax;
    const Real lor = fast_div(sp.lorA, axr * axr + sp.g2);
    if (CHI == CHI_NONE) return lor;
    if (sizeof(Real) == 8) return lor * (Real)chi_factor_d<CHI>(ax, lv);
    return lor * (Real)chi_factor_f<CHI>(ax, (float)ax, lv);
  }
  return voigt_core<Real, CHI>(Xd, sp.qx, sp.vy, sp.lorA, sp.g2, sp.hum, lv.perrin_b1, lv.perrin_b2, c.sqrt14);
}

// Classification of one line against subinterval [s, se] (LBL.f90:81-98 and
// the first tests of leftLBL / rightLBL): returns the distance D >= 1 from
// the line to the nearest grid-0 position and whether the line sits left of
// the subinterval; false when the line is near, inside or beyond the cutoff.
__device__ __forceinline__ bool far_line(double nu, double s, double se, double cut, double &D,
                                         bool &left) {
  if (nu < s) {
    D = -(nu - s);
    left = true;
    return !(D > cut) && !(D < 1.0);
  }
  if (nu > se) {
    D = (nu - s) - DELTA_WV;
    left = false;
    return !(D >= cut) && !(D < 1.0);
  }
  return false;
}

// upper end of the UU (or V) interval of centre lines that walk over cell j
// of grid k: (2*floor((j+1)/2) + 2) * H_k  (derived from LineGridCalc.f90:202-331)
__device__ __forceinline__ double walk_hi(int j, double hk) { return (double)(2 * ((j + 1) / 2) + 2) * hk; }

// Bounds of the near lines of subinterval [s, se] in a level's shifted-centre
// order: which = 0 first line with nu' > s - 1 (or inside), 1 first with
// nu' >= s, 2 first with nu' > se, 3 first line at least 1 cm-1 right of the
// subinterval.  [b0, b1) near-left, [b1, b2) centre, [b2, b3) near-right.
// Found by one warp: each step probes 32 evenly spaced positions of the
// remaining range at once (the predicate is monotone: false ... true), so
// that about four dependent loads replace a binary search's eighteen.  Every
// lane of the warp calls it and gets the result.
__device__ __forceinline__ int64_t near_bound_warp(const double *snu, int64_t n, double s, double se, int which) {
  const int lane = threadIdx.x & 31;
  auto pred = [&](double v) {
    if (which == 0) return !(v < s && (v - s) <= -1.0);
    if (which == 1) return v >= s;
    if (which == 2) return v > se;
    return v > se && ((v - s) - DELTA_WV) >= 1.0;
  };
  int64_t lo = 0, hi = n; // the answer lies in [lo, hi]
  while (hi - lo > 32) {
    const int64_t span = hi - lo;
    const int64_t pos = lo + (span * (lane + 1)) / 33; // in [lo, hi)
    const unsigned b = __ballot_sync(0xffffffffu, pred(snu[pos]));
    if (b) {
      const int f = __ffs(b) - 1;
      const int64_t pf = lo + (span * (f + 1)) / 33;
      const int64_t pp = f > 0 ? lo + (span * f) / 33 + 1 : lo;
      lo = pp;
      hi = pf;
    } else {
      lo = lo + (span * 32) / 33 + 1;
    }
  }
  const int64_t pos = lo + lane;
  const unsigned b = __ballot_sync(0xffffffffu, pos < hi && pred(snu[pos]));
  return b ? lo + (__ffs(b) - 1) : hi;
}

// Whether near line `li` (shifted centre v) contributes to the subinterval:
// inside the line window, within the cutoff (left side keeps D == cutoff,
// right side drops it: LineGridCalc.f90:23, 509), centre lines with UU < 10.
// Sets UU = v - s and the class (0 near-left, 1 centre, 2 near-right).
__device__ __forceinline__ bool near_keep(double v, int64_t li, double s, double se, double cut, int64_t wlo,
                                          int64_t whi, double &UU, int &cls) {
  UU = v - s;
  cls = 1;
  if (li < wlo || li >= whi) return false;
  if (v < s) { cls = 0; return -UU <= cut; }
  if (v > se) { cls = 2; return (UU - DELTA_WV) < cut; }
  return UU < DELTA_WV;
}

// Far-line sums of grid-0 cell J of one unit over its far-kernel chunks
// [c0, c1): P(J), M(J), L(J) and the RK(1) position, for the 32 lanes of one
// warp (lanes over chunks, then a fixed-order xor reduction: every lane gets
// the same sums, in the same order for every call).
__device__ __forceinline__ void far_cell_sums(const double *far, int c0, int c1, int J, double (&f)[4]) {
  f[0] = f[1] = f[2] = f[3] = 0.0;
  for (int c = c0 + (int)(threadIdx.x & 31); c < c1; c += 32) {
    f[0] += far[(size_t)c * NFAR + 2 * (J - 1)];
    f[1] += far[(size_t)c * NFAR + 2 * J - 1];
    f[2] += far[(size_t)c * NFAR + 2 * J];
    f[3] += far[(size_t)c * NFAR];
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int i = 0; i < 4; ++i) f[i] += __shfl_xor_sync(0xffffffffu, f[i], off);
}

// Far-line sums of grid-0 cell J of one unit: read from the unit's folded
// row (its far-kernel chunks summed per position by far_fold_kernel) when
// there is one, else summed here over the chunks.
__device__ __forceinline__ void far_sums(const double *fold, const double *far, int c0, int c1, int J,
                                         double (&f)[4]) {
  if (fold) {
    f[0] = fold[2 * (J - 1)];
    f[1] = fold[2 * J - 1];
    f[2] = fold[2 * J];
    f[3] = fold[0];
  } else {
    far_cell_sums(far, c0, c1, J, f);
  }
}

} // namespace marfa
