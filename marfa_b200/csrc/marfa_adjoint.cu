// marfa_adjoint.cu -- vector-Jacobian products of the PT records (FP64).
//
// For a cotangent g on the records of every (level, subinterval), the VJP of
// L = sum g * record is returned with respect to the level temperatures and
// pressures and the per-line reference intensity S and air broadening
// gamma_air.  The forward accumulators are recomputed by the FP64 kernels of
// marfa_kernels.cu; nothing of the line shape is stored.  Per unit:
//
//   cascade_adjoint_kernel  recomputes the cascade (Grids.f90:80-139) of one
//                           grid-0 subtree with its clamp decisions and runs it
//                           backwards: dL/d(accumulator) for every P, M, L
//                           slot and direct finest point (the cascade is
//                           piecewise linear, the clamp weights are fixed by
//                           the forward decisions);
//   near_adjoint_kernel     one thread per near line: every (slot, X) pair of
//                           the reference schedule (centerLBL, and the fine
//                           parts of leftLBL / rightLBL), the line shape and
//                           its partial derivatives by forward-mode dual
//                           numbers, weighted by the slot gradients;
//   far_adjoint_kernel      one thread per far line: the 21 grid-0 positions.
//
// Per (line, unit) the weighted sums of the shape and its partials are turned
// into the four gradients by the chain rule through the per-line
// spectroscopy (Spectroscopy.f90:38-145), whose partial derivatives
// adjoint_prep_kernel evaluates once per (level, line).  The placement of a
// line (which cells it walks) depends on the shifted centre discontinuously
// and is held fixed, as are the Humlicek region choices and the clamp
// decisions: the VJP is the derivative of the piecewise-smooth map.
#include <type_traits>
#include "marfa_kernels.cuh"

namespace marfa {

// ---------------------------------------------------------- dual numbers
// Value and partial derivatives with respect to (|X|, alpha_D, gamma_L, T).
struct Dual {
  double v, d[4];
};
__device__ __forceinline__ Dual dconst(double c) { return {c, {0.0, 0.0, 0.0, 0.0}}; }
__device__ __forceinline__ Dual dvar(double x, int i) {
  Dual r = dconst(x);
  r.d[i] = 1.0;
  return r;
}
__device__ __forceinline__ Dual operator+(const Dual &a, const Dual &b) {
  Dual r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
__device__ __forceinline__ Dual operator-(const Dual &a, const Dual &b) {
  Dual r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
__device__ __forceinline__ Dual operator*(const Dual &a, const Dual &b) {
  Dual r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
__device__ __forceinline__ Dual operator/(const Dual &a, const Dual &b) {
  Dual r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
__device__ __forceinline__ Dual operator+(const Dual &a, double c) { Dual r = a; r.v += c; return r; }
__device__ __forceinline__ Dual operator+(double c, const Dual &a) { return a + c; }
__device__ __forceinline__ Dual operator-(const Dual &a, double c) { Dual r = a; r.v -= c; return r; }
__device__ __forceinline__ Dual operator-(double c, const Dual &a) {
  Dual r;
  r.v = c - a.v;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = -a.d[i];
  return r;
}
__device__ __forceinline__ Dual operator*(const Dual &a, double c) {
  Dual r;
  r.v = a.v * c;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] * c;
  return r;
}
__device__ __forceinline__ Dual operator*(double c, const Dual &a) { return a * c; }
__device__ __forceinline__ Dual operator/(double c, const Dual &b) { return dconst(c) / b; }
__device__ __forceinline__ Dual operator/(const Dual &a, double c) { return a * (1.0 / c); }
__device__ __forceinline__ Dual dexp(const Dual &a) {
  Dual r;
  r.v = exp(a.v);
#pragma unroll
  for (int i = 0; i < 4; ++i) r.d[i] = a.d[i] * r.v;
  return r;
}
__device__ __forceinline__ Dual dhorner_acc(Dual acc, const Dual &) { return acc; }
template <typename... Rest>
__device__ __forceinline__ Dual dhorner_acc(Dual acc, const Dual &x, double c, Rest... rest) {
  return dhorner_acc(acc * x + c, x, rest...);
}
template <typename... Rest>
__device__ __forceinline__ Dual dhorner(const Dual &x, double c0, Rest... rest) {
  return dhorner_acc(dconst(c0), x, rest...);
}

// chi-factors of ChiFactors.f90:29-122 with |X| (and, for perrin, T) as
// dual variables; pieces decided on the value of |X| as in chi_factor_d.
template <int CHI>
__device__ Dual chi_dual(const Dual &ax, const Dual &T) {
  if (CHI == CHI_TONKOV) {
    if (ax.v > 3.0) {
      if (ax.v <= 150.0) return 1.084 * dexp(-0.027 * ax);
      if (ax.v <= 300.0) return 0.208 * dexp(-0.016 * ax);
      return 0.025 * dexp(-0.009 * ax);
    }
  } else if (CHI == CHI_POLLACK) {
    if (ax.v >= 3.0) {
      if (ax.v < 10.0) return 1.35 * dexp(-1.0 * ax / 10.0);
      return 0.614 * dexp(-1.0 * ax / 47.0);
    }
  } else if (CHI == CHI_PERRIN) {
    if (ax.v > 3.0) {
      const Dual b1 = 0.0888 - 0.16 * dexp(-0.00410 * T);
      const Dual b2 = 0.0526 * dexp(-0.00152 * T);
      const double b3 = 0.0232;
      if (ax.v < 30.0) return dexp(-1.0 * (b1 * (ax - 3.0)));
      if (ax.v < 120.0) return dexp(-1.0 * (b1 * 27.0) - b2 * (ax - 30.0));
      return dexp(-1.0 * (b1 * 27.0) - b2 * 90.0 - b3 * (ax - 120.0));
    }
  }
  return dconst(1.0);
}

// The line shape per unit intensity, G = F / S(T), with its partials with
// respect to (|X|, alpha_D, gamma_L, T): the regions and formulas of
// Shapes.f90:22-133 and Spectroscopy.f90:194-261 evaluated on dual numbers.
// Region decisions use the same double values as the forward shape
// (VX = |X| * (sqln2 / alpha), VY = sqln2 * gamma / alpha).
template <int CHI>
__device__ Dual shape_dual(double ax_v, double alpha, double gamma, double T_v, const Consts &c) {
  const Dual ax = dvar(ax_v, 0), A = dvar(alpha, 1), Gm = dvar(gamma, 2), T = dvar(T_v, 3);
  const Dual qx = c.sqln2 / A;
  const Dual VX = ax * qx;
  const Dual VY = (c.sqln2 * Gm) / A;
  const double VXd = VX.v, VYd = VY.v;
  const Dual lorA = Gm / c.pi;
  const Dual g2 = Gm * Gm;
  const Dual hum = c.sqln2 / (c.sqrtpi * A);
  if (VXd >= 15.0) return lorA / (ax * ax + g2) * chi_dual<CHI>(ax, T);
  const Dual x = VX * VX;
  const double sum = VXd + VYd;
  if (sum >= 15.0) {
    const Dual Y = VY, Y2 = Y * Y;
    const Dual A1 = (0.2820948 + 0.5641896 * Y2) * Y;
    const Dual B1 = 0.5641896 * Y;
    const Dual A2 = 0.25 + Y2 + Y2 * Y2;
    const Dual B2 = Y2 + Y2 - 1.0;
    return (A1 + B1 * x) / (A2 + B2 * x + x * x) * hum;
  }
  if (sum >= 5.5) {
    const Dual Y = VY, Y2 = Y * Y;
    const Dual A3 = Y * dhorner(Y2, 0.56419, 3.10304, 4.65456, 1.05786);
    const Dual B3 = Y * dhorner(Y2, 1.69257, 0.56419, 2.962);
    const Dual C3 = Y * (1.69257 * Y2 - 2.53885);
    const Dual D3 = Y * 0.56419;
    const Dual A4 = dhorner(Y2, 1.0, 6.0, 10.5, 4.5, 0.5625);
    const Dual B4 = dhorner(Y2, 4.0, 6.0, 9.0, -4.5);
    const Dual C4 = 10.5 + 6.0 * (Y2 - 1.0) * Y2;
    const Dual D4 = 4.0 * Y2 - 6.0;
    return (((D3 * x + C3) * x + B3) * x + A3) / ((((x + D4) * x + C4) * x + B4) * x + A4) * hum;
  }
  if (VXd <= 1.0 || VYd >= 0.02) {
    const Dual Y = VY;
    const Dual A5 = dhorner(Y, 0.564224, 7.55895, 49.5213, 204.510, 581.746, 1174.8, 1678.33, 1629.76, 973.778,
                            272.102);
    const Dual B5 = dhorner(Y, 2.25689, 22.6778, 100.705, 247.198, 336.364, 220.843, -2.34403, -60.5644);
    const Dual C5 = dhorner(Y, 3.38534, 22.6798, 52.8454, 42.5683, 18.546, 4.58029);
    const Dual D5 = dhorner(Y, 2.25689, 7.56186, 1.66203, -0.128922);
    const Dual E5 = dhorner(Y, 0.564224, 0.971457E-3);
    const Dual A6 = dhorner(Y, 1.0, 13.3988, 88.2674, 369.199, 1074.41, 2256.98, 3447.63, 3764.97, 2802.87,
                            1280.83, 272.102);
    const Dual B6 = dhorner(Y, 5., 53.5952, 266.299, 793.427, 1549.68, 2037.31, 1758.34, 902.306, 211.678);
    const Dual C6 = dhorner(Y, 10., 80.3928, 269.292, 479.258, 497.302, 308.186, 78.866);
    const Dual D6 = dhorner(Y, 10., 53.5952, 92.7586, 55.0293, 22.0353);
    const Dual E6 = dhorner(Y, 5.0, 13.3988, 1.49645);
    return ((((E5 * x + D5) * x + C5) * x + B5) * x + A5) /
           (((((x + E6) * x + D6) * x + C6) * x + B6) * x + A6) * hum;
  }
  if (VXd > 5.0) return lorA / (ax * ax + g2) * chi_dual<CHI>(ax, T) * (1.0 + 1.5 / x);
  const Dual dop = hum * dexp(-1.0 * x);
  if (VXd > c.sqrt14) {
    const double Ut[9] = {1., 1.5, 2., 2.5, 3., 3.5, 4., 4.5, 5.};
    const double Wt[9] = {-0.688, 0.2667, 0.6338, 0.4405, 0.2529, 0.1601, 0.1131, 0.0853, 0.068};
    int I = (int)(VXd / 0.5 - 1.00001);
    I = I < 1 ? 1 : (I > 8 ? 8 : I);
    const Dual F = 2.0 * (Wt[I - 1] * (Ut[I] - VX) + Wt[I] * (VX - Ut[I - 1]));
    return dop + lorA / (ax * ax) * (1.0 + F);
  }
  return dop;
}

// Weighted sums over the evaluations of one line in one unit.
struct LineSums {
  double a0, ax, al, ga, t; // sum g*G, g*dG/dnu' (through X), g*dG/dalpha, g*dG/dgamma, g*dG/dT
  __device__ void init() { a0 = ax = al = ga = t = 0.0; }
  // one evaluation at offset X with dX/dnu' = sgn, weighted by g
  template <int CHI>
  __device__ __forceinline__ void add(double g, double X, double sgn, double alpha, double gamma, double T,
                                      const Consts &c) {
    if (g == 0.0) return;
    const Dual G = shape_dual<CHI>(fabs(X), alpha, gamma, T, c);
    const double sx = X > 0.0 ? 1.0 : (X < 0.0 ? -1.0 : 0.0);
    a0 += g * G.v;
    ax += g * G.d[0] * sx * sgn;
    al += g * G.d[1];
    ga += g * G.d[2];
    t += g * G.d[3];
  }
};

// --------------------------------------------------- per-line chain rule
// Partial derivatives of the per-(level, line) spectroscopy of prep_kernel.
__global__ void __launch_bounds__(256) adjoint_prep_kernel(AdjPrepParams p) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int l = blockIdx.y;
  if (i >= p.lines.n) return;
  const LevelConst lv = p.lv[l];
  const Consts c = p.c;
  const size_t o = (size_t)l * p.lines.n + i;
  LineAux a;
  a.ratio = 0.0;
  a.dlnS_dT = 0.0;
  a.dg_dT = a.dg_dP = a.dg_dgair = 0.0;
  a.delta = (double)p.lines.delta[i];
  const int iso = p.lines.iso[i];
  if (iso >= 1 && iso <= p.n_iso) {
    const double T = lv.T, P = lv.P;
    const double nair = (double)p.lines.nair[i];
    const double gair = p.lines.gair64 ? p.lines.gair64[i] : (double)p.lines.gair[i];
    const double gself = (double)p.lines.gself[i];
    const double tf = pow(c.tref / T, nair);
    a.dg_dgair = tf * (P - lv.pself);
    a.dg_dP = tf * gair;
    // pself = n 10 k T / p0 grows with T at fixed number density
    const double gamma = tf * (gair * (P - lv.pself) + gself * lv.pself);
    a.dg_dT = -nair / T * gamma + tf * (gself - gair) * (lv.pself / T);
    int idx = 1;
    double uw = 0.0;
    if (tips_node(T, p.tgrid, p.n_temp, idx, uw)) {
      const double *row = p.tips + (size_t)(iso - 1) * p.n_temp;
      const double lw = 1.0 - uw;
      const double Q = lw * row[idx - 1] + uw * row[idx];
      const double dQ = (row[idx] - row[idx - 1]) / p.tgrid.dt;
      const double Qref = tips_ref(row, p.tgrid, p.n_temp);
      const double E = (double)p.lines.elow[i];
      const double nu = p.lines.nu[i];
      const double boltz = exp(-(c.c2 * E / T)) / exp(-(c.c2 * E / c.tref));
      const double en = exp(-(c.c2 * nu / T));
      const double emis = (1.0 - en) / (1.0 - exp(-(c.c2 * nu / c.tref)));
      a.ratio = (Qref / Q) * boltz * emis;
      a.dlnS_dT = -dQ / Q + c.c2 * E / (T * T) - en * (c.c2 * nu / (T * T)) / (1.0 - en);
    }
  }
  p.aux[o] = a;
}

// ------------------------------------------------------- cascade adjoint
__device__ __forceinline__ void quarter_w(double near_edge, double mid, double far_edge, double (&w)[3]) {
  const double A = 0.375 * near_edge + 0.75 * mid - 0.125 * far_edge;
  if (A < near_edge || A < mid) { w[0] = 0.5; w[1] = 0.5; w[2] = 0.0; }
  else { w[0] = 0.375; w[1] = 0.75; w[2] = -0.125; }
}

__device__ __forceinline__ double quarter_v(double near_edge, double mid, double far_edge) {
  double A = 0.375 * near_edge + 0.75 * mid - 0.125 * far_edge;
  if (A < near_edge || A < mid) A = 0.5 * (near_edge + mid);
  return A;
}

// offset (in cells) of grid k inside one grid-0 subtree: 2^k - 1
__device__ __forceinline__ int sub_off(int k) { return (1 << k) - 1; }

__global__ void __launch_bounds__(256) cascade_adjoint_kernel(CascadeAdjParams p) {
  const int ub = blockIdx.x / NT0;
  const int J = blockIdx.x - ub * NT0 + 1;
  const int u = p.unit0 + ub;
  const int l = u / p.n_sub, sub = u - l * p.n_sub;
  const double *scr = p.scratch + (size_t)ub * SCR_STRIDE;
  double *gs = p.gscratch + (size_t)ub * SCR_STRIDE;
  __shared__ double val[1023 * 3]; // forward cell values of the subtree, grid k at sub_off(k)
  __shared__ double gv[1023 * 3];  // their gradients
  if (threadIdx.x < 32) { // grid-0 cell J as cascade_kernel forms it
    double f[4];
    far_sums(p.fold ? p.fold + ((size_t)l * p.n_sub + sub) * NFAR : nullptr,
             p.far + ((size_t)l * p.n_chunks) * NFAR, p.sub_chunk0[sub], p.sub_chunk0[sub + 1], J, f);
    if (threadIdx.x == 0) {
      val[0] = f[0] + scr[1 + J - 1];
      val[1] = f[1] + scr[11 + J - 1];
      val[2] = f[2] + scr[21 + J - 1];
    }
  }
  __syncthreads();
  // forward cascade, as cascade_kernel (same operations, same decisions)
  for (int k = 1; k <= 9; ++k) {
    const int ncell = 1 << k;
    const int cb = base_k(k) - NT0 + (J - 1) * ncell;
    const double *prev = val + 3 * sub_off(k - 1);
    double *cur = val + 3 * sub_off(k);
    for (int t = threadIdx.x; t < ncell; t += blockDim.x) {
      const int pt = t >> 1;
      const double cP = prev[3 * pt], cM = prev[3 * pt + 1], cL = prev[3 * pt + 2];
      double P = scr[SCR_FINE_P + cb + t], M = scr[SCR_FINE_M + cb + t], L = scr[SCR_FINE_L + cb + t];
      if ((t & 1) == 0) { P += cP; M += quarter_v(cP, cM, cL); L += cM; }
      else { P += cM; M += quarter_v(cL, cM, cP); L += cL; }
      cur[3 * t] = P;
      cur[3 * t + 1] = M;
      cur[3 * t + 2] = L;
    }
    __syncthreads();
  }
  const double dens = p.target == 1 ? p.lv[l].density : 1.0;
  const size_t rec = ((size_t)(p.level_out0 + l) * p.n_sub + sub) * NT;
  // finest points RK(4j-2 .. 4j+1) of grid-9 cell j
  {
    const double *v9 = val + 3 * sub_off(9);
    double *g9 = gv + 3 * sub_off(9);
    const int cb = base_k(9) - NT0 + (J - 1) * 512;
    for (int t = threadIdx.x; t < 512; t += blockDim.x) {
      const double cP = v9[3 * t], cM = v9[3 * t + 1], cL = v9[3 * t + 2];
      const int j = (J - 1) * 512 + t + 1;
      double g[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int i = 4 * j - 2 + q;
        g[q] = p.cot[rec + i - 1] * dens;
        gs[SCR_RK + i - 2] = g[q];
      }
      double w[3], w2[3];
      quarter_w(cP, cM, cL, w);
      quarter_w(cL, cM, cP, w2);
      const double gP = g[0] * w[0] + g[2] * w2[2];
      const double gM = g[0] * w[1] + g[1] + g[2] * w2[1];
      const double gL = g[0] * w[2] + g[2] * w2[0] + g[3];
      g9[3 * t] = gP;
      g9[3 * t + 1] = gM;
      g9[3 * t + 2] = gL;
      gs[SCR_FINE_P + cb + t] = gP;
      gs[SCR_FINE_M + cb + t] = gM;
      gs[SCR_FINE_L + cb + t] = gL;
    }
  }
  __syncthreads();
  // grid k+1 -> grid k (k = 8 .. 0): each parent gathers its two children
  for (int k = 8; k >= 0; --k) {
    const int ncell = 1 << k;
    const double *vk = val + 3 * sub_off(k);
    const double *gc = gv + 3 * sub_off(k + 1);
    double *gk = gv + 3 * sub_off(k);
    for (int t = threadIdx.x; t < ncell; t += blockDim.x) {
      const double cP = vk[3 * t], cM = vk[3 * t + 1], cL = vk[3 * t + 2];
      double w[3], w2[3];
      quarter_w(cP, cM, cL, w);   // even child: M += quarter(cP, cM, cL)
      quarter_w(cL, cM, cP, w2);  // odd child:  M += quarter(cL, cM, cP)
      const double eP = gc[6 * t], eM = gc[6 * t + 1], eL = gc[6 * t + 2];
      const double oP = gc[6 * t + 3], oM = gc[6 * t + 4], oL = gc[6 * t + 5];
      const double gP = eP + eM * w[0] + oM * w2[2];
      const double gM = eM * w[1] + eL + oP + oM * w2[1];
      const double gL = eM * w[2] + oM * w2[0] + oL;
      gk[3 * t] = gP;
      gk[3 * t + 1] = gM;
      gk[3 * t + 2] = gL;
      if (k >= 1) {
        const int cb = base_k(k) - NT0 + (J - 1) * ncell;
        gs[SCR_FINE_P + cb + t] = gP;
        gs[SCR_FINE_M + cb + t] = gM;
        gs[SCR_FINE_L + cb + t] = gL;
      } else {
        gs[1 + J - 1] = gP;
        gs[11 + J - 1] = gM;
        gs[21 + J - 1] = gL;
      }
    }
    __syncthreads();
  }
  if (J == 1 && threadIdx.x == 0) gs[0] = p.cot[rec] * dens;
}

// ------------------------------------------------ chain rule and reduction
// Turns the weighted sums of one (line, unit) into the per-line gradients
// (atomic, a line meets many units) and this thread's share of the level's.
__device__ __forceinline__ void line_chain(const LineSums &a, const LineGen &g, const LineAux &x, double nus,
                                           double T, int64_t li, const AdjointParams &p, double &tT,
                                           double &tP) {
  if (a.a0 == 0.0 && a.ax == 0.0 && a.al == 0.0 && a.ga == 0.0 && a.t == 0.0) return;
  const double S = g.S;
  atomicAdd(p.dS + li, x.ratio * a.a0);
  atomicAdd(p.dgair + li, S * a.ga * x.dg_dgair);
  tT += S * (a.a0 * x.dlnS_dT + a.al * (g.alpha / (2.0 * T)) + a.ga * x.dg_dT + a.t);
  tP += S * (a.ga * x.dg_dP + a.al * (g.alpha * x.delta / nus) + a.ax * x.delta);
}

__device__ __forceinline__ void level_reduce_add(double tT, double tP, double *dT, double *dP) {
  __shared__ double red[2][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    tT += __shfl_down_sync(0xffffffffu, tT, off);
    tP += __shfl_down_sync(0xffffffffu, tP, off);
  }
  if (lane == 0) { red[0][warp] = tT; red[1][warp] = tP; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sT = 0.0, sP = 0.0;
    for (int w = 0; w < nw; ++w) { sT += red[0][w]; sP += red[1][w]; }
    if (sT != 0.0) atomicAdd(dT, sT);
    if (sP != 0.0) atomicAdd(dP, sP);
  }
}

// --------------------------------------------------------- near lines
// Every evaluation of near line (UU, cls) in the reference schedule, as
// emit(slotA, slotB, X, dX/dnu'): one shape value added to accumulator slots
// A and B (B < 0: none) of the unit's scratch layout.  The conditions are the
// placement rules of fine_kernel (derived from LineGridCalc.f90:7-674) seen
// from the line: for each grid only the few cells whose conditions can hold
// are tested, with the same double comparisons.
template <class Emit>
__device__ void near_line_walk(double UU, int cls, Emit &&emit) {
  const double U = UU - DELTA_WV, V = DELTA_WV - UU;
  // grid 0 and RK(1) (as grid0_line)
  {
    const int n0 = UU >= 2.0 ? (int)floor(UU) - 1 : 0;
    const int m0 = V >= 2.0 ? (int)floor(V) - 1 : 0;
    for (int e = 0; e <= 10; ++e) {
      bool toL = false, toP = false;
      double X = 0.0, sg = 1.0;
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
        else if (e >= 10 - m0) { toP = e <= 9; toL = e >= 11 - m0; X = V - (double)(10 - e); sg = -1.0; }
      }
      if (toL || toP) {
        const int sa = toL ? (e == 0 ? 0 : 21 + e - 1) : -1;
        const int sb = (toP && e <= 9) ? 1 + e : -1;
        emit(sa, sb, X, sg);
      }
    }
    for (int m = 1; m <= 10; ++m) {
      bool on = false;
      double X = 0.0, sg = 1.0;
      if (cls == 0) { on = m >= 2; X = (UU - (double)(m - 1)) - 0.5; }
      else if (cls == 2) { on = m <= 9; X = (U + (double)(10 - m)) + 0.5; }
      else if (m <= n0) { on = true; X = (UU - (double)m) + 0.5; }
      else if (m >= 11 - m0) { on = true; X = (V - (double)(11 - m)) + 0.5; sg = -1.0; }
      if (on) emit(11 + m - 1, -1, X, sg);
    }
  }
  // grids 1..9
  for (int k = 1; k <= 9; ++k) {
    const double hk = h_k(k), hk1 = h_k(k - 1), hn = h_k(k + 1);
    const int ntk = nt_k(k);
    const int cb = base_k(k) - NT0;
    auto sP = [&](int e) { return SCR_FINE_P + cb + e; };     // P(e+1)
    auto sL = [&](int e) { return SCR_FINE_L + cb + e - 1; }; // L(e)
    auto sM = [&](int m) { return SCR_FINE_M + cb + m - 1; }; // M(m)
    if (cls == 1) {
      const int n = (int)floor(UU / hk);
      for (int e = max(0, n - 4); e <= min(ntk, n); ++e) { // left walk, edges
        const bool hasL = e >= 1, hasP = e <= ntk - 1;
        const bool tl = hasL && UU >= (double)(e + 1) * hk && UU < walk_hi(e, hk);
        const bool tp = hasP && UU >= (double)(e + 2) * hk && UU < walk_hi(e + 1, hk);
        if (tl || tp) emit(tl ? sL(e) : -1, tp ? sP(e) : -1, UU - (double)e * hk, 1.0);
      }
      const int nv = (int)floor(V / hk);
      for (int e = max(0, ntk - nv); e <= min(ntk, ntk - nv + 4); ++e) { // right walk, edges
        const bool hasL = e >= 1, hasP = e <= ntk - 1;
        const int rL = ntk + 1 - e, rP = ntk - e;
        const bool tl = hasL && V >= (double)(rL + 1) * hk && V < walk_hi(rL, hk);
        const bool tp = hasP && V >= (double)(rP + 1) * hk && V < walk_hi(rP, hk);
        if (tl || tp) emit(tl ? sL(e) : -1, tp ? sP(e) : -1, V - (double)rP * hk, -1.0);
      }
      for (int m = max(1, n - 3); m <= min(ntk, n); ++m) // left walk, mids
        if (UU >= (double)(m + 1) * hk && UU < walk_hi(m, hk)) emit(sM(m), -1, (UU - (double)m * hk) + hn, 1.0);
      for (int m = max(1, ntk + 1 - nv); m <= min(ntk, ntk + 4 - nv); ++m) { // right walk, mids
        const int r = ntk + 1 - m;
        if (V >= (double)(r + 1) * hk && V < walk_hi(r, hk))
          emit(sM(m), -1, ((DELTA_WV - UU) - (double)r * hk) + hn, -1.0);
      }
    } else if (cls == 0) {
      if (UU > -hk1) { // D = -UU < H_{k-1}: cells 1 and 2
        const bool own = -UU >= hk;
        if (own) emit(-1, sP(0), UU, 1.0);
        emit(own ? sL(1) : -1, sP(1), UU - hk, 1.0);
        emit(sL(2), -1, UU - hk1, 1.0);
        if (own) emit(sM(1), -1, UU - hn, 1.0);
        emit(sM(2), -1, (UU - hk) - hn, 1.0);
      }
    } else {
      if (U < hk1) { // cells ntk and ntk - 1
        const bool own = U >= hk;
        if (own) emit(sL(ntk), -1, U, 1.0);
        emit(sL(ntk - 1), own ? sP(ntk - 1) : -1, U + hk, 1.0);
        emit(-1, sP(ntk - 2), U + hk1, 1.0);
        if (own) emit(sM(ntk), -1, U + hn, 1.0);
        emit(sM(ntk - 1), -1, (U + hk) + hn, 1.0);
      }
    }
  }
  // direct finest points RK(i), i = 2..NT
  const double H = HSTEP, H9 = h_k(9);
  if (cls == 1) {
    const int ni = (int)floor(UU / H);
    for (int i = max(2, ni - 7); i <= min(NT, ni + 1); ++i) { // left fine loop
      const double xi = (double)(i - 1) * H;
      if (UU >= xi && UU < (double)(4 * ((i - 2) / 4) + 8) * H) emit(SCR_RK + i - 2, -1, UU - xi, 1.0);
    }
    for (int i = max(2, ni + 1); i <= min(NT, ni + 10); ++i) { // right fine loop
      const double xi = (double)(i - 1) * H;
      if (UU < xi && V < (double)((NT - i) / 4 + 2) * H9) emit(SCR_RK + i - 2, -1, UU - xi, 1.0);
    }
  } else if (cls == 0) {
    if (UU > -H9) {
      emit(SCR_RK + 0, -1, UU - H, 1.0);
      emit(SCR_RK + 1, -1, (UU - H) - H, 1.0);
      emit(SCR_RK + 2, -1, (UU + H) - H9, 1.0);
      emit(SCR_RK + 3, -1, UU - H9, 1.0);
    }
  } else {
    if (U < H9) {
      emit(SCR_RK + NT - 2, -1, U, 1.0);
      emit(SCR_RK + NT - 3, -1, U + H, 1.0);
      emit(SCR_RK + NT - 4, -1, (U + H) + H, 1.0);
      emit(SCR_RK + NT - 5, -1, (U + H9) - H, 1.0);
    }
  }
}

template <int CHI>
__global__ void __launch_bounds__(256) near_adjoint_kernel(AdjointParams p) {
  const int ub = blockIdx.y;
  const int u = p.unit0 + ub;
  const int l = u / p.win.n_sub, sub = u - l * p.win.n_sub;
  const double *snu = p.snu + (size_t)l * p.n_lines;
  const int *sidx = p.sidx + (size_t)l * p.n_lines;
  const double s = p.win.sub_s[sub], se = p.win.sub_e[sub];
  const double *gs = p.gscratch + (size_t)ub * SCR_STRIDE;
  const LevelConst lv = p.lv[l];
  __shared__ int64_t sb[4];
  if (threadIdx.x < 128) { // warp w finds bound w
    const int64_t v = near_bound_warp(snu, p.n_lines, s, se, threadIdx.x >> 5);
    if ((threadIdx.x & 31) == 0) sb[threadIdx.x >> 5] = v;
  }
  __syncthreads();
  const int64_t a = sb[0], b = sb[3];
  double tT = 0.0, tP = 0.0;
  for (int64_t q = a + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < b; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t li = sidx[q];
    double UU;
    int cls;
    if (!near_keep(snu[q], li, s, se, p.cutoff, p.win.lo[sub], p.win.hi[sub], UU, cls)) continue;
    const size_t o = (size_t)l * p.n_lines + li;
    const LineGen g = p.gen[o];
    LineSums acc;
    acc.init();
    near_line_walk(UU, cls, [&](int sa, int sbb, double X, double sg) {
      const double w = (sa >= 0 ? gs[sa] : 0.0) + (sbb >= 0 ? gs[sbb] : 0.0);
      acc.add<CHI>(w, X, sg, g.alpha, g.gamma, lv.T, p.c);
    });
    line_chain(acc, g, p.aux[o], snu[q], lv.T, li, p, tT, tP);
  }
  level_reduce_add(tT, tP, p.dT + p.level_out0 + l, p.dP + p.level_out0 + l);
}

// ----------------------------------------------------------- far lines
template <int CHI>
__global__ void __launch_bounds__(256) far_adjoint_kernel(AdjointParams p) {
  const int ub = blockIdx.y;
  const int u = p.unit0 + ub;
  const int l = u / p.win.n_sub, sub = u - l * p.win.n_sub;
  const int ci = p.sub_chunk0[sub] + blockIdx.x;
  if (ci >= p.sub_chunk0[sub + 1]) return; // uniform over the block
  const double *gs = p.gscratch + (size_t)ub * SCR_STRIDE;
  const LevelConst lv = p.lv[l];
  // gradient of each grid-0 position: integer position e feeds RK(1) (e = 0),
  // P(e+1) and L(e); half-integer position m - 1/2 feeds M(m)
  __shared__ double gpos[NFAR];
  if (threadIdx.x < NFAR) {
    const int t = threadIdx.x;
    double w;
    if ((t & 1) == 0) {
      const int e = t / 2;
      w = (e == 0 ? gs[0] : 0.0) + (e <= 9 ? gs[1 + e] : 0.0) + (e >= 1 ? gs[21 + e - 1] : 0.0);
    } else {
      w = gs[11 + (t + 1) / 2 - 1];
    }
    gpos[t] = w;
  }
  __syncthreads();
  const double s = p.win.sub_s[sub], se = p.win.sub_e[sub];
  const size_t lo = (size_t)l * p.n_lines;
  double tT = 0.0, tP = 0.0;
  for (int64_t i = p.chunk_begin[ci] + threadIdx.x; i < p.chunk_end[ci]; i += blockDim.x) {
    double D;
    bool left;
    const double nus = p.nus[lo + i];
    if (!far_line(nus, s, se, p.cutoff, D, left)) continue;
    const LineGen g = p.gen[lo + i];
    LineSums acc;
    acc.init();
    // left line: X = D + k/2 at position k, D = s - nu'; right line: position 20 - k
    for (int k = 0; k < NFAR; ++k)
      acc.add<CHI>(gpos[left ? k : NFAR - 1 - k], D + 0.5 * k, left ? -1.0 : 1.0, g.alpha, g.gamma, lv.T, p.c);
    line_chain(acc, g, p.aux[lo + i], nus, lv.T, i, p, tT, tP);
  }
  level_reduce_add(tT, tP, p.dT + p.level_out0 + l, p.dP + p.level_out0 + l);
}

// ------------------------------------------------------------ launchers
cudaError_t launch_adjoint_prep(const AdjPrepParams &p, cudaStream_t st) {
  if (p.lines.n == 0) return cudaSuccess;
  dim3 grid((unsigned)((p.lines.n + 255) / 256), (unsigned)p.n_levels);
  adjoint_prep_kernel<<<grid, 256, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_cascade_adjoint(const CascadeAdjParams &p, cudaStream_t st) {
  if (p.n_units <= 0) return cudaSuccess;
  cascade_adjoint_kernel<<<p.n_units * NT0, 256, 0, st>>>(p);
  return cudaGetLastError();
}

template <int CHI>
static void line_adjoint_dispatch(const AdjointParams &p, int near_blocks, cudaStream_t st) {
  near_adjoint_kernel<CHI><<<dim3((unsigned)near_blocks, (unsigned)p.n_units), 256, 0, st>>>(p);
  if (p.max_chunks > 0)
    far_adjoint_kernel<CHI><<<dim3((unsigned)p.max_chunks, (unsigned)p.n_units), 256, 0, st>>>(p);
}

cudaError_t launch_line_adjoint(const AdjointParams &p, int chi, int near_blocks, cudaStream_t st) {
  if (p.n_units <= 0) return cudaSuccess;
  near_blocks = near_blocks < 1 ? 1 : near_blocks;
  switch (chi) {
    case CHI_TONKOV: line_adjoint_dispatch<CHI_TONKOV>(p, near_blocks, st); break;
    case CHI_POLLACK: line_adjoint_dispatch<CHI_POLLACK>(p, near_blocks, st); break;
    case CHI_PERRIN: line_adjoint_dispatch<CHI_PERRIN>(p, near_blocks, st); break;
    default: line_adjoint_dispatch<CHI_NONE>(p, near_blocks, st); break;
  }
  return cudaGetLastError();
}

} // namespace marfa
