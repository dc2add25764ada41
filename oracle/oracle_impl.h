/*
 * oracle_impl.h -- body of the CPU oracle, compiled twice (TEST INFRASTRUCTURE).
 *
 * Included by oracle_mixed.c (ORACLE_TYPEMAP_MIXED=1) and oracle_fp64.c
 * (ORACLE_TYPEMAP_MIXED=0).  `real` is the Fortran default real of the
 * reference; every promotion to double below mirrors a mixed-kind expression
 * in the reference (Fortran evaluates real*real(DP) in DP).  In the fp64 map
 * real == double and the casts vanish.
 *
 * Restated from (file:line in the reference project):
 *   Constants.f90:4-23            constants (float parameters in the reference)
 *   Spectroscopy.f90:38-145       shift, Doppler/Lorentz HWHM, TIPS, S(T)
 *   Spectroscopy.f90:194-261      lorentz, doppler, chi-corrected lorentz,
 *                                 region-4 asymptotics
 *   ChiFactors.f90:18-122         none / tonkov / pollack / perrin
 *   Shapes.f90:22-133             Humlicek-Kuntz voigt (regions 0-4)
 *   LineGridCalc.f90:7-179        leftLBL
 *   LineGridCalc.f90:181-494      centerLBL
 *   LineGridCalc.f90:496-674      rightLBL
 *   Grids.f90:64-139              reset, interpolation_step, cascade
 *   LBL.f90:25-100                line window loop (lblScheme)
 *   main.f90:81-180, 196-248      level / subinterval loops, starting line
 *
 * The reference keeps all state in module globals; here it lives in a
 * per-level work struct so levels can run in parallel.
 */
#include <math.h>
#include <string.h>
#include <stdlib.h>
#include <stdint.h>
#include "marfa_oracle.h"

#if ORACLE_TYPEMAP_MIXED
typedef float real;
#define RL(x) x##f
#define r_sqrt sqrtf
#define r_exp expf
#define r_pow powf
#define SFX(n) n##_mixed
#else
typedef double real;
#define RL(x) x
#define r_sqrt sqrt
#define r_exp exp
#define r_pow pow
#define SFX(n) n##_fp64
#endif

/* ---- grid geometry: Grids.f90:6-16, 20, 48-58 ------------------------- */
#define NT0 10
#define NT 20481
#define NCELLS 10230
static inline int nt_k(int k) { return NT0 << k; }
static inline int base_k(int k) { return NT0 * ((1 << k) - 1); }
/* H_k = 2^-k (k = 0..9), H = H9/4; H_10 is written H+H in the reference. */
static const double HK[11] = {1.0, 0.5, 0.25, 0.125, 0.0625, 0.03125, 0.015625,
                              0.0078125, 0.00390625, 0.001953125, 0.0009765625};
#define HF 0.00048828125 /* H */
#define DELTA_WV 10.0

/* ---- constants: Constants.f90 (float parameters folded at compile time) */
typedef struct {
  real PI, SQLN2, C2, DOPPLER, TREF, BOLSI, STDP, SQRTPI, SQRT14, LOG2;
} consts_t;

static consts_t SFX(make_consts)(void) {
  consts_t c;
#if ORACLE_TYPEMAP_MIXED
  /* gfortran folds parameter expressions with correct rounding at the kind's
   * precision, one operation at a time; float arithmetic reproduces that. */
  float log2f_ = (float)0.69314718055994530942; /* nearest float to ln 2 */
  float planck = 6.626070e-27f, spl = 2.99792458e10f, bolsgs = 1.3806503e-16f;
  float avo = 6.02214076e23f;
  float t;
  c.PI = 3.1415926f;
  c.LOG2 = log2f_;
  c.SQLN2 = sqrtf(log2f_);
  t = planck * spl;
  c.C2 = t / bolsgs;
  t = 2.0f * avo;
  t = t * bolsgs;
  t = t * log2f_;
  t = sqrtf(t);
  c.DOPPLER = t / spl;
  c.TREF = 296.0f;
  c.BOLSI = 1.3806503e-23f;
  c.STDP = 101325.0f;
  c.SQRTPI = sqrtf(c.PI);
  c.SQRT14 = sqrtf(1.4f);
#else
  c.PI = 3.1415926;
  c.LOG2 = log(2.0);
  c.SQLN2 = sqrt(log(2.0));
  c.C2 = 6.626070e-27 * 2.99792458e10 / 1.3806503e-16;
  c.DOPPLER = sqrt(2.0 * 6.02214076e23 * 1.3806503e-16 * log(2.0)) / 2.99792458e10;
  c.TREF = 296.0;
  c.BOLSI = 1.3806503e-23;
  c.STDP = 101325.0;
  c.SQRTPI = sqrt(c.PI);
  c.SQRT14 = sqrt(1.4);
#endif
  return c;
}

/* ---- per-level work state (the reference's module globals) ------------ */
typedef struct {
  consts_t c;
  /* current line (Spectroscopy.f90:18-32) */
  real lineIntensity, dopHWHM, lorHWHM;
  /* run / level settings */
  int chi, shape, molcode;
  real temperature;
  real cutoff;
  /* region-1..3 coefficient caches (Shapes.f90:45-47 `save`); recomputed
   * whenever VY changes, which is semantically neutral */
  real Y1, Y2, Y3;
  real A1, B1, A2, B2, A3, B3, C3, D3, A4, B4, C4, D4;
  real A5, B5, C5, D5, E5, A6, B6, C6, D6, E6;
  int64_t evals;
  int64_t negative_shape; /* F < 0 would trigger the EPS early returns */
  int last_region;
  /* grids */
  real P[NCELLS], M[NCELLS], L[NCELLS];
  real RK[NT];
} work_t;

/* ---- chi factors: ChiFactors.f90:18-122 ------------------------------- */
static real SFX(chi_factor)(const work_t *w, double X) {
  const int code = w->molcode;
  double ax = fabs(X);
  switch (w->chi) {
  case ORACLE_CHI_TONKOV: { /* ChiFactors.f90:29-53 */
    real f = RL(1.);
    if (code == 2) {
      if (ax > 3.0) {
        if (ax <= 150.0) f = (real)((double)RL(1.084) * exp(-((double)RL(0.027) * ax)));
        else if (ax <= 300.0) f = (real)((double)RL(0.208) * exp(-((double)RL(0.016) * ax)));
        else f = (real)((double)RL(0.025) * exp(-((double)RL(0.009) * ax)));
      }
    }
    return f;
  }
  case ORACLE_CHI_POLLACK: { /* ChiFactors.f90:55-80 */
    real f = RL(1.);
    if (code == 2) {
      if (ax >= 3.0) {
        if (ax < 10.0) f = (real)((double)RL(1.35) * exp(-ax / 10.0));
        else f = (real)((double)RL(0.614) * exp(-ax / 47.0));
      }
    }
    return f;
  }
  case ORACLE_CHI_PERRIN: { /* ChiFactors.f90:82-122 */
    real f = RL(1.);
    const real T = w->temperature;
    real B1 = RL(0.0888) - RL(0.16) * r_exp(-(RL(0.00410) * T));
    real B2 = RL(0.0526) * r_exp(-(RL(0.00152) * T));
    real B3 = RL(0.0232);
    real S1 = RL(3.), S2 = RL(30.), S3 = RL(120.);
    if (code == 2) {
      if (ax > (double)S1) {
        if (ax < (double)S2) {
          f = (real)exp(-((double)B1 * (ax - (double)S1)));
        } else if (ax < (double)S3) {
          f = (real)exp((double)(-(B1 * (S2 - S1))) - (double)B2 * (ax - (double)S2));
        } else {
          f = (real)exp((double)(-(B1 * (S2 - S1)) - B2 * (S3 - S2)) -
                        (double)B3 * (ax - (double)S3));
        }
      }
    }
    return f;
  }
  default:
    return RL(1.); /* noneChi, ChiFactors.f90:18-27 */
  }
}

/* lorentz(X, gamma) * S, Spectroscopy.f90:194-203 (evaluated in DP) */
static real SFX(lorentz)(const work_t *w, double X, real g) {
  double den = X * X + (double)(real)(g * g);
  double v = (double)g / ((double)w->c.PI * den) * (double)w->lineIntensity;
  return (real)v;
}
/* doppler(X, alpha) * S, Spectroscopy.f90:206-215 */
static real SFX(doppler)(const work_t *w, double X, real a) {
  real pre = w->c.SQLN2 / (w->c.SQRTPI * a);
  double q = X / (double)a;
  double e = exp(-((q * q) * (double)w->c.LOG2));
  return (real)((double)pre * e * (double)w->lineIntensity);
}
/* Spectroscopy.f90:218-229 */
static real SFX(chi_lorentz)(const work_t *w, double X, real g) {
  real l = SFX(lorentz)(w, X, g);
  real f = SFX(chi_factor)(w, X);
  return l * f;
}

/* Humlicek-Kuntz voigt with the reference's region 0 and region-4
 * asymptotics, Shapes.f90:22-133 and Spectroscopy.f90:232-261. */
static real SFX(voigt)(work_t *w, double X) {
  const real alpha = w->dopHWHM, gam = w->lorHWHM, S = w->lineIntensity;
  real VX = (real)fabs((double)w->c.SQLN2 * X / (double)alpha);
  real VY = w->c.SQLN2 * gam / alpha;
  real VXs, v;
  if (VX >= RL(15.)) { /* region 0 */
    w->last_region = 0;
    return SFX(chi_lorentz)(w, X, gam);
  }
  VXs = VX * VX;
  if (VX + VY >= RL(15.0)) { /* region 1 */
    if (VY != w->Y1) {
      real Y_2;
      w->Y1 = VY;
      Y_2 = w->Y1 * w->Y1;
      w->A1 = (RL(0.2820948) + RL(0.5641896) * Y_2) * w->Y1;
      w->B1 = RL(0.5641896) * w->Y1;
      w->A2 = RL(0.25) + Y_2 + Y_2 * Y_2;
      w->B2 = Y_2 + Y_2 - RL(1.);
    }
    v = (w->A1 + w->B1 * VXs) / (w->A2 + w->B2 * VXs + VXs * VXs);
    w->last_region = 1;
    return v / w->c.SQRTPI / (alpha / w->c.SQLN2) * S;
  } else if (VX + VY >= RL(5.5)) { /* region 2 */
    if (VY != w->Y2) {
      real Y_2;
      w->Y2 = VY;
      Y_2 = w->Y2 * w->Y2;
      w->A3 = w->Y2 * (((RL(0.56419) * Y_2 + RL(3.10304)) * Y_2 + RL(4.65456)) * Y_2 + RL(1.05786));
      w->B3 = w->Y2 * ((RL(1.69257) * Y_2 + RL(0.56419)) * Y_2 + RL(2.962));
      w->C3 = w->Y2 * (RL(1.69257) * Y_2 - RL(2.53885));
      w->D3 = w->Y2 * RL(0.56419);
      w->A4 = (((Y_2 + RL(6.0)) * Y_2 + RL(10.5)) * Y_2 + RL(4.5)) * Y_2 + RL(0.5625);
      w->B4 = ((RL(4.0) * Y_2 + RL(6.0)) * Y_2 + RL(9.0)) * Y_2 - RL(4.5);
      w->C4 = RL(10.5) + RL(6.0) * (Y_2 - RL(1.0)) * Y_2;
      w->D4 = RL(4.0) * Y_2 - RL(6.0);
    }
    v = (((w->D3 * VXs + w->C3) * VXs + w->B3) * VXs + w->A3) /
        ((((VXs + w->D4) * VXs + w->C4) * VXs + w->B4) * VXs + w->A4);
    w->last_region = 2;
    return v / w->c.SQRTPI / (alpha / w->c.SQLN2) * S;
  } else if (VX <= RL(1.0) || VY >= RL(0.02)) { /* region 3 */
    if (VY != w->Y3) {
      real Y3;
      w->Y3 = VY;
      Y3 = w->Y3;
      w->A5 = ((((((((RL(0.564224) * Y3 + RL(7.55895)) * Y3 + RL(49.5213)) * Y3 + RL(204.510)) * Y3 +
                  RL(581.746)) * Y3 + RL(1174.8)) * Y3 + RL(1678.33)) * Y3 + RL(1629.76)) * Y3 +
               RL(973.778)) * Y3 + RL(272.102);
      w->B5 = ((((((RL(2.25689) * Y3 + RL(22.6778)) * Y3 + RL(100.705)) * Y3 + RL(247.198)) * Y3 +
                RL(336.364)) * Y3 + RL(220.843)) * Y3 - RL(2.34403)) * Y3 - RL(60.5644);
      w->C5 = ((((RL(3.38534) * Y3 + RL(22.6798)) * Y3 + RL(52.8454)) * Y3 + RL(42.5683)) * Y3 +
               RL(18.546)) * Y3 + RL(4.58029);
      w->D5 = ((RL(2.25689) * Y3 + RL(7.56186)) * Y3 + RL(1.66203)) * Y3 - RL(0.128922);
      w->E5 = RL(0.971457E-3) + RL(0.564224) * Y3;
      w->A6 = (((((((((Y3 + RL(13.3988)) * Y3 + RL(88.2674)) * Y3 + RL(369.199)) * Y3 + RL(1074.41)) * Y3 +
                   RL(2256.98)) * Y3 + RL(3447.63)) * Y3 + RL(3764.97)) * Y3 + RL(2802.87)) * Y3 +
               RL(1280.83)) * Y3 + RL(272.102);
      w->B6 = (((((((RL(5.) * Y3 + RL(53.5952)) * Y3 + RL(266.299)) * Y3 + RL(793.427)) * Y3 +
                 RL(1549.68)) * Y3 + RL(2037.31)) * Y3 + RL(1758.34)) * Y3 + RL(902.306)) * Y3 +
              RL(211.678);
      w->C6 = (((((RL(10.) * Y3 + RL(80.3928)) * Y3 + RL(269.292)) * Y3 + RL(479.258)) * Y3 +
                RL(497.302)) * Y3 + RL(308.186)) * Y3 + RL(78.866);
      w->D6 = (((RL(10.) * Y3 + RL(53.5952)) * Y3 + RL(92.7586)) * Y3 + RL(55.0293)) * Y3 + RL(22.0353);
      w->E6 = (RL(5.0) * Y3 + RL(13.3988)) * Y3 + RL(1.49645);
    }
    v = ((((w->E5 * VXs + w->D5) * VXs + w->C5) * VXs + w->B5) * VXs + w->A5) /
        (((((VXs + w->E6) * VXs + w->D6) * VXs + w->C6) * VXs + w->B6) * VXs + w->A6);
    w->last_region = 3;
    return v / w->c.SQRTPI / (alpha / w->c.SQLN2) * S;
  } else { /* region 4 */
    if (VX > RL(5.)) { /* voigtAsymptotic1, Spectroscopy.f90:232-242 */
      real l = SFX(chi_lorentz)(w, X, gam);
      w->last_region = 40;
      return l * (RL(1.) + RL(1.5) / (VX * VX));
    } else if (VX > w->c.SQRT14) { /* voigtAsymptotic2, Spectroscopy.f90:245-261 */
      static const real U[9] = {RL(1.), RL(1.5), RL(2.), RL(2.5), RL(3.), RL(3.5), RL(4.), RL(4.5), RL(5.)};
      static const real W[9] = {RL(-0.688), RL(0.2667), RL(0.6338), RL(0.4405), RL(0.2529),
                                RL(0.1601), RL(0.1131), RL(0.0853), RL(0.068)};
      int I = (int)(VX / RL(0.5) - RL(1.00001)); /* 1-based, truncation */
      real F = RL(2.) * (W[I - 1] * (U[I] - VX) + W[I] * (VX - U[I - 1]));
      real d = SFX(doppler)(w, X, alpha);
      double t = (double)gam / ((double)w->c.PI * (X * X)) * (double)(RL(1.) + F) * (double)S;
      w->last_region = 41;
      return (real)((double)d + t);
    } else {
      w->last_region = 42;
      return SFX(doppler)(w, X, alpha);
    }
  }
}

/* FSHAPE: shapeFuncPtr => voigt (Shapes.f90:11-15) or lorentzShape
 * (Shapes.f90:135-141: chiCorrectedLorentz(X, lorHWHM)), plus two diagnostic
 * shapes used by placement tests (constant 1, and |X|). */
static inline real SFX(fshape)(work_t *w, double X) {
  real v;
  w->evals++;
  if (w->shape == ORACLE_SHAPE_ONE) return RL(1.);
  if (w->shape == ORACLE_SHAPE_ABSX) return (real)fabs(X);
  if (w->shape == ORACLE_SHAPE_LORENTZ) return SFX(chi_lorentz)(w, X, w->lorHWHM);
  v = SFX(voigt)(w, X);
  if (v < RL(0.)) w->negative_shape++;
  return v;
}
#define FSH(x) SFX(fshape)(w, (x))
#define GP(k, j) w->P[base_k(k) + (j) - 1]
#define GM(k, j) w->M[base_k(k) + (j) - 1]
#define GL(k, j) w->L[base_k(k) + (j) - 1]
#define RKI(i) w->RK[(i) - 1]
/* H_{k+1} as the reference writes it: H+H for the grid-9 mid point. */
static inline double hnext(int k) { return k == 9 ? (HF + HF) : HK[k + 1]; }

/* ---- leftLBL: LineGridCalc.f90:7-179 ------------------------------------
 * Line left of the subinterval; UU = nu' - start < 0.  EPS is 0 for the whole
 * run (Grids.f90:66) and shapes are non-negative, so the `FF < EPS` exits are
 * kept only as counted events (negative_shape). */
static void SFX(left_lbl)(work_t *w, double freq, double ul) {
  double UU = ul - freq, XXX;
  real FF;
  int k, kk, i;
  if (UU >= 0.) return;
  if (-UU > (double)w->cutoff) return;
  FF = FSH(UU);
  if (FF < (real)0) return;
  RKI(1) = FF + RKI(1);
  if (!(-UU < HK[0])) { /* the whole grid 0 */
    GP(0, 1) += FF;
    FF = FSH(UU - HK[1]);
    GM(0, 1) += FF;
    FF = FSH(UU - HK[0]);
    GL(0, 1) += FF;
    goto grid0;
  }
  for (k = 1; k <= 9; ++k)
    if (!(-UU < HK[k])) break;
  if (k <= 9) { /* H_k <= -UU < H_{k-1}: cell 1 of grid k */
    GP(k, 1) += FF;
    FF = (k == 9) ? FSH(UU - HF - HF) : FSH(UU - HK[k + 1]);
    GM(k, 1) += FF;
    FF = FSH(UU - HK[k]);
    GL(k, 1) += FF;
    if (FF < (real)0) return;
  } else { /* -UU < H9: finest points 2..5 directly */
    RKI(2) = RKI(2) + FSH(UU - HF);
    RKI(3) = RKI(3) + FSH(UU - HF - HF);
    RKI(4) = RKI(4) + FSH(UU + HF - HK[9]);
    FF = FSH(UU - HK[9]);
    RKI(5) = RKI(5) + FF;
    k = 9;
  }
  /* cascade: cell 2 of grids k..1 (labels 12k .. 121) */
  for (kk = k; kk >= 1; --kk) {
    GP(kk, 2) += FF;
    FF = (kk == 9) ? FSH(UU - HK[9] - HF - HF) : FSH(UU - HK[kk] - HK[kk + 1]);
    GM(kk, 2) += FF;
    FF = FSH(UU - HK[kk - 1]);
    GL(kk, 2) += FF;
    if (kk >= 2 && kk <= 8 && FF < (real)0) return;
  }
grid0: /* label 10: grid 0 cells 2..10 */
  XXX = HK[0];
  for (i = 2; i <= NT0; ++i) {
    GP(0, i) += FF;
    FF = FSH(UU - XXX - HK[1]);
    GM(0, i) += FF;
    XXX = XXX + HK[0];
    FF = FSH(UU - XXX);
    GL(0, i) += FF;
    if (FF < (real)0) return;
  }
}

/* ---- rightLBL: LineGridCalc.f90:496-674 -------------------------------- */
static void SFX(right_lbl)(work_t *w, double freq, double ul) {
  double UU = ul - freq - DELTA_WV, XXX;
  real FF;
  int k, kk, i, n;
  if (UU >= (double)w->cutoff) return;
  FF = FSH(UU);
  if (FF < (real)0) return;
  if (!(UU < HK[0])) {
    GL(0, NT0) += FF;
    FF = FSH(UU + HK[1]);
    GM(0, NT0) += FF;
    FF = FSH(UU + HK[0]);
    GP(0, NT0) += FF;
    goto grid0;
  }
  for (k = 1; k <= 9; ++k)
    if (!(UU < HK[k])) break;
  if (k <= 8) { /* labels 60..67 then 13k */
    n = nt_k(k);
    GL(k, n) += FF;
    FF = FSH(UU + HK[k + 1]);
    GM(k, n) += FF;
    FF = FSH(UU + HK[k]);
    GP(k, n) += FF;
    if (FF < (real)0) return;
    kk = k;
  } else {
    if (k == 9) { /* label 68 */
      n = nt_k(9);
      GL(9, n) += FF;
      FF = FSH(UU + HF + HF);
      GM(9, n) += FF;
      FF = FSH(UU + HK[9]);
      GP(9, n) += FF;
      if (FF < (real)0) return;
    } else { /* label 69: UU < H9 */
      RKI(NT) = RKI(NT) + FSH(UU);
      RKI(NT - 1) = RKI(NT - 1) + FSH(UU + HF);
      RKI(NT - 2) = RKI(NT - 2) + FSH(UU + HF + HF);
      RKI(NT - 3) = RKI(NT - 3) + FSH(UU + HK[9] - HF);
    }
    /* label 139: grid 9 cell NT9-1, with the first shape call repeated */
    n = nt_k(9) - 1;
    FF = FSH(UU + HK[9]);
    GL(9, n) += FF;
    FF = FSH(UU + HK[9] + HF + HF);
    GM(9, n) += FF;
    FF = FSH(UU + HK[8]);
    GP(9, n) += FF;
    kk = 8;
  }
  for (; kk >= 1; --kk) { /* labels 13kk: cell NT_kk - 1 */
    n = nt_k(kk) - 1;
    GL(kk, n) += FF;
    FF = FSH(UU + HK[kk] + HK[kk + 1]);
    GM(kk, n) += FF;
    FF = FSH(UU + HK[kk - 1]);
    GP(kk, n) += FF;
    if (kk <= 8 && kk >= 2 && FF < (real)0) return;
  }
grid0: /* label 12: grid 0 cells 9..1, then RK(1) */
  XXX = HK[0];
  for (i = NT0 - 1; i >= 1; --i) {
    GL(0, i) += FF;
    FF = FSH(UU + XXX + HK[1]);
    GM(0, i) += FF;
    XXX = XXX + HK[0];
    FF = FSH(UU + XXX);
    GP(0, i) += FF;
    if (FF < (real)0) return;
  }
  RKI(1) = RKI(1) + FF;
}

/* ---- centerLBL: LineGridCalc.f90:181-494 ------------------------------- */
static void SFX(center_lbl)(work_t *w, double freq, double ul) {
  double UU = ul - freq, CONSER, UUU;
  real FF, FA;
  int npoint, i, k, I, III, ib, icon, ii, done;
  if (UU >= DELTA_WV) return;
  FF = FSH(0.0);
  if (FF < (real)0) return;
  npoint = 1;
  CONSER = UU - HF;
  FA = FSH(UU);
  if (FA > (real)0) RKI(1) = RKI(1) + FA; /* EPS4 = 0.25*EPS = 0 */
  if (UU >= HF) {
    /* left side: walk from the subinterval start toward the line, one grid
     * per pass, finer as the remaining distance UUU shrinks (labels 201-209) */
    I = 0;
    UUU = UU;
    for (k = 0; k <= 9; ++k) {
      if (k > 0) I = I * 2;
      if (k == 0 ? (UUU < HK[0] + HK[0]) : (UUU < HK[k - 1])) continue;
      done = 0;
      for (i = I + 1; i <= nt_k(k); ++i) {
        UUU = UUU - HK[k];
        FF = FSH(UUU);
        if (!(FF < (real)0)) {
          GP(k, i) += FA;
          GM(k, i) += FSH(UUU + hnext(k));
          GL(k, i) += FF;
        }
        FA = FF;
        if (UUU - HK[k] < HK[k]) { I = i; done = 1; break; }
      }
      if (!done) I = nt_k(k); /* not reachable for UU < 10 */
    }
    /* label 210: finest points from the last grid-9 edge up to the line */
    I = I * 4;
    ib = I + 2;
    CONSER = UU - (double)((real)(ib - 1) * (real)HF); /* integer*real -> real */
    for (icon = ib; icon <= NT; ++icon) {
      RKI(icon) = RKI(icon) + FSH(CONSER);
      CONSER = CONSER - HF;
      if (CONSER < 0.) break;
    }
    if (icon > NT) return; /* GOTO 11: not reachable for UU < 10 */
    npoint = icon;
  }
  /* label 211: right side, walking from the subinterval end toward the line */
  npoint = npoint + 1;
  UUU = DELTA_WV - UU;
  FA = FSH(UUU);
  III = 0;
  for (k = 0; k <= 9; ++k) {
    if (k > 0) III = III * 2;
    if (k == 0 ? (UUU < HK[0] + HK[0]) : (UUU < HK[k - 1])) continue;
    done = 0;
    for (i = nt_k(k) - III; i >= 1; --i) {
      III = III + 1;
      UUU = UUU - HK[k];
      FF = FSH(UUU);
      if (!(FF < (real)0)) {
        GL(k, i) += FA;
        GM(k, i) += FSH(UUU + hnext(k));
        GP(k, i) += FF;
      }
      FA = FF;
      if (UUU - HK[k] < HK[k]) { done = 1; break; }
    }
    (void)done;
  }
  /* label 310: finest points from just right of the line to the first
   * right-side grid-9 edge */
  III = III * 4;
  I = NT - III;
  for (ii = npoint; ii <= I; ++ii) {
    RKI(ii) = RKI(ii) + FSH(CONSER);
    CONSER = CONSER - HF;
  }
}

/* ---- interpolation_step / cascadeInterpolation: Grids.f90:80-139 ------- */
static void SFX(cascade)(work_t *w) {
  int k, J, I, n;
  for (k = 0; k < 9; ++k) {
    const int bc = base_k(k), bf = base_k(k + 1);
    n = nt_k(k);
    for (J = 1; J <= n; ++J) {
      real cP = w->P[bc + J - 1], cM = w->M[bc + J - 1], cL = w->L[bc + J - 1], A;
      I = 2 * J - 1;
      w->P[bf + I - 1] += cP;
      A = RL(0.375) * cP + RL(0.75) * cM - RL(0.125) * cL;
      if (A < cP || A < cM) A = RL(0.5) * (cP + cM);
      w->M[bf + I - 1] += A;
      w->L[bf + I - 1] += cM;
      I = I + 1;
      w->P[bf + I - 1] += cM;
      A = RL(0.375) * cL + RL(0.75) * cM - RL(0.125) * cP;
      if (A < cL || A < cM) A = RL(0.5) * (cL + cM);
      w->M[bf + I - 1] += A;
      w->L[bf + I - 1] += cL;
    }
  }
  {
    const int b9 = base_k(9);
    I = 1;
    for (J = 1; J <= nt_k(9); ++J) {
      real cP = w->P[b9 + J - 1], cM = w->M[b9 + J - 1], cL = w->L[b9 + J - 1], A;
      I = I + 1;
      A = cP * RL(0.375) + cM * RL(0.75) - cL * RL(0.125);
      if (A < cP || A < cM) A = RL(0.5) * (cP + cM);
      RKI(I) = RKI(I) + A;
      I = I + 1;
      RKI(I) = RKI(I) + cM;
      I = I + 1;
      A = cL * RL(0.375) + cM * RL(0.75) - cP * RL(0.125);
      if (A < cL || A < cM) A = RL(0.5) * (cL + cM);
      RKI(I) = RKI(I) + A;
      I = I + 1;
      RKI(I) = RKI(I) + cL;
    }
  }
}

/* ---- line record (LBL.f90:43-44; processParFile.f90:140-176) ----------- */
typedef struct {
  double nu;
  real S, gair, gself, E, nair, delta;
  int32_t jmi;
} line_t;

static void SFX(read_line)(const unsigned char *rec, line_t *ln) {
  float f[5], d;
  memcpy(&ln->nu, rec, 8);
  memcpy(f, rec + 8, 20);
  memcpy(&ln->jmi, rec + 28, 4);
  memcpy(&d, rec + 32, 4);
  ln->S = (real)f[0];
  ln->gair = (real)f[1];
  ln->gself = (real)f[2];
  ln->E = (real)f[3];
  ln->nair = (real)f[4];
  ln->delta = (real)d;
}

/* Isotopologue masses WISO(124), MolarMasses.f90:9-145 (generated data table
 * shared with the library). */
#include "marfa_wiso.h"
#if ORACLE_TYPEMAP_MIXED
#define ORACLE_WISO MARFA_WISO_F
#else
#define ORACLE_WISO MARFA_WISO_D
#endif

typedef struct {
  real pressure, temperature, density, pSelf;
} level_t;

/* per-line spectroscopy: LBL.f90:64-73 with Spectroscopy.f90:38-145 */
static int SFX(prepare_line)(work_t *w, const oracle_args *a, const level_t *lv,
                             const line_t *ln, double *nu_shift) {
  const consts_t *c = &w->c;
  int iso = ln->jmi / 100;
  real molar, T = lv->temperature, Q, Qref, tips_factor, boltz, emis, lwt, lw, uw, tval, t0, dt;
  double k296;
  int idx;
  double nus;
  if (iso < 1 || iso > MARFA_WISO_LEN || iso > a->n_iso) return 13;
  molar = (real)ORACLE_WISO[iso - 1];
  /* shiftedLinePosition: real*real product promoted to DP */
  nus = ln->nu + (double)(real)(ln->delta * lv->pressure);
  *nu_shift = nus;
  /* dopplerHWHM: DP product, real sqrt(T/M) */
  w->dopHWHM = (real)((double)c->DOPPLER * nus * (double)r_sqrt(T / molar));
  /* lorentzHWHM */
  w->lorHWHM = r_pow(c->TREF / T, ln->nair) *
               (ln->gair * (lv->pressure - lv->pSelf) + ln->gself * lv->pSelf);
  /* TIPSofT on the table's grid; on the reference's (20 K, 2 K) these are
   * its operations: tval = (T - 20) / 2 + 1, lwt = idx * 2 + 18, and
   * Q(296) = TIPS(iso, 139) */
  t0 = (real)a->tips_t0;
  dt = (real)a->tips_dt;
  tval = (T - t0) / dt + RL(1.);
  if (!(tval >= RL(1.)) || !(tval < (real)a->n_temp)) return 11;
  idx = (int)tval;
  lwt = (real)(idx - 1) * dt + t0;
  uw = (T - lwt) / dt;
  lw = RL(1.) - uw;
  Q = lw * (real)a->tips[(size_t)(iso - 1) * a->n_temp + (idx - 1)] +
      uw * (real)a->tips[(size_t)(iso - 1) * a->n_temp + idx];
  k296 = (a->tips_dt > 0.0) ? (296.0 - a->tips_t0) / a->tips_dt : -1.0;
  if (k296 >= 0.0 && k296 == (double)(int)k296 && (int)k296 < a->n_temp) {
    Qref = (real)a->tips[(size_t)(iso - 1) * a->n_temp + (int)k296];
  } else { /* 296 K between two nodes */
    real tr = (RL(296.) - t0) / dt + RL(1.);
    int ir = (int)tr;
    real ur = (RL(296.) - ((real)(ir - 1) * dt + t0)) / dt;
    Qref = (RL(1.) - ur) * (real)a->tips[(size_t)(iso - 1) * a->n_temp + (ir - 1)] +
           ur * (real)a->tips[(size_t)(iso - 1) * a->n_temp + ir];
  }
  /* intensityOfT (uses the unshifted nu) */
  tips_factor = Qref / Q;
  boltz = r_exp(-(c->C2 * ln->E / T)) / r_exp(-(c->C2 * ln->E / c->TREF));
  emis = (real)((1.0 - exp(-((double)c->C2 * ln->nu / (double)T))) /
                (1.0 - exp(-((double)c->C2 * ln->nu / (double)c->TREF))));
  w->lineIntensity = ln->S * tips_factor * boltz * emis;
  return 0;
}

/* ---- one atmospheric level: main.f90:86-174 with lblScheme LBL.f90:25-100.
 * Subintervals run in order; `dump_sub` >= 0 stops after that subinterval's
 * line loop and copies the raw accumulators out. */
static int SFX(run_level)(const oracle_args *a, int lev, int64_t start_idx, double start_line_wv,
                          float *out, double *out64, int64_t *evals, int dump_sub, double *dump) {
  work_t *w = (work_t *)calloc(1, sizeof(work_t));
  level_t lv;
  const unsigned char *recs = (const unsigned char *)a->records;
  int nsub = oracle_num_subintervals(a->start_wv, a->end_wv), isub = 0, rc = 0;
  double s, e;
  int64_t line_idx = start_idx;
  if (!w) return 10;
  w->c = SFX(make_consts)();
  w->chi = a->chi;
  w->shape = a->shape;
  w->molcode = a->mol_code;
  w->cutoff = (real)a->cutoff;
  w->Y1 = w->Y2 = w->Y3 = (real)0;
  lv.pressure = (real)a->pressure[lev];
  lv.temperature = (real)a->temperature[lev];
  lv.density = (real)a->density[lev];
  lv.pSelf = lv.density * RL(10.) * w->c.BOLSI * lv.temperature / w->c.STDP;
  w->temperature = lv.temperature;
  s = a->start_wv;
  e = s + DELTA_WV;
  while (s < a->end_wv) {
    double ext_end = s + DELTA_WV + (double)w->cutoff;
    double cap = (s - (double)w->cutoff) + DELTA_WV;
    int64_t I;
    if (cap <= start_line_wv) cap = start_line_wv;
    memset(w->P, 0, sizeof w->P);
    memset(w->M, 0, sizeof w->M);
    memset(w->L, 0, sizeof w->L);
    memset(w->RK, 0, sizeof w->RK);
    for (I = line_idx;; ++I) { /* LBL_LOOP */
      line_t ln;
      double nus;
      if (I > a->n_lines) { rc = 9; goto done; } /* reference would loop forever */
      SFX(read_line)(recs + (size_t)(I - 1) * 36, &ln);
      if (ln.nu >= ext_end) break;
      if (ln.nu <= cap) line_idx = I;
      rc = SFX(prepare_line)(w, a, &lv, &ln, &nus);
      if (rc) goto done;
      if (nus < s) SFX(left_lbl)(w, s, nus);
      else if (nus > e) SFX(right_lbl)(w, s, nus);
      else SFX(center_lbl)(w, s, nus);
    }
    if (isub == dump_sub) {
      int j;
      for (j = 0; j < NT; ++j) dump[j] = (double)w->RK[j];
      for (j = 0; j < NCELLS; ++j) {
        dump[NT + j] = (double)w->P[j];
        dump[NT + NCELLS + j] = (double)w->M[j];
        dump[NT + 2 * NCELLS + j] = (double)w->L[j];
      }
      goto done;
    }
    SFX(cascade)(w);
    if (out || out64) {
      size_t off = ((size_t)lev * nsub + isub) * NT;
      int j;
      for (j = 0; j < NT; ++j) {
        real v = (a->target == ORACLE_TARGET_VAC) ? lv.density * w->RK[j] : w->RK[j];
        if (out) out[off + j] = (float)v;
        if (out64) out64[off + j] = (double)v;
      }
    }
    s = s + DELTA_WV;
    e = s + DELTA_WV;
    ++isub;
  }
done:
  if (evals) *evals = w->evals;
  free(w);
  return rc;
}

/* shape value probe for tests */
static int SFX(shape_probe)(const oracle_args *a, int lev, int64_t line, double X, double *value,
                            int *region) {
  work_t *w = (work_t *)calloc(1, sizeof(work_t));
  level_t lv;
  line_t ln;
  double nus;
  int rc;
  if (!w) return 10;
  w->c = SFX(make_consts)();
  w->chi = a->chi;
  w->shape = a->shape;
  w->molcode = a->mol_code;
  lv.pressure = (real)a->pressure[lev];
  lv.temperature = (real)a->temperature[lev];
  lv.density = (real)a->density[lev];
  lv.pSelf = lv.density * RL(10.) * w->c.BOLSI * lv.temperature / w->c.STDP;
  w->temperature = lv.temperature;
  SFX(read_line)((const unsigned char *)a->records + (size_t)line * 36, &ln);
  rc = SFX(prepare_line)(w, a, &lv, &ln, &nus);
  if (!rc) {
    *value = (double)SFX(fshape)(w, X);
    if (region) *region = w->last_region;
  }
  free(w);
  return rc;
}
