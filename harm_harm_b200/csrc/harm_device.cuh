// harm_device.cuh -- per-point device physics of the GRMHD step (sm_100a).
//
// Templated on the arithmetic type T: the flux path (state, fluxes, wave speeds) runs in
// T = float for the mixed-precision step and T = double for the FP64 step; the
// conserved update, source terms and the inversion always run in double.
//
// Reference formulas (HARM, WHICHVEL=VELREL4, REMOVERESTMASSFROMUU=2, PRIMMAXWELL):
//   ucon from relative 4-velocity ....... phys.tools.c:1900 (ucon_calc_rel4vel_fromuconrel)
//   1+u_t ............................... phys.tools.c:1272 (compute_1plusud0_rel4vel)
//   b^2 ................................. phys.tools.c:1392 (bsq_calc_fromq_rel4vel)
//   fluxes / conserved .................. phys.tools.c:30, :1071, :1133, :392
//   fast speeds ......................... vchar.c:34, simplefast vchar.c:260
//   connection source ................... phys.c:132 (source_conn)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "harm_b200.h"

namespace hb {

constexpr int NPR = HARM_NPR;

// One metric record in registers.  Symmetric tensors as 10 entries 00,01,02,03,11,12,13,22,23,33.
template <typename T>
struct Geo {
  T gcov[10], gcon[10];
  T gcovpert_tt, alpha, betasqoalphasq, beta1, beta2, beta3, gdet, igdet;
};

__host__ __device__ constexpr int sym(int m, int n) {
  return (m <= n) ? ((m == 0) ? n : (m == 1) ? 3 + n : (m == 2) ? 5 + n : 9)
                  : ((n == 0) ? m : (n == 1) ? 3 + m : (n == 2) ? 5 + m : 9);
}

// Load a record from a plane-major table tab[field][plane] at 2-D offset c: a read-only
// global table (LDG), or a copy staged in shared memory (plain loads).
template <bool LDG, typename S>
__device__ __forceinline__ S tab_ld(const S* p) {
  if constexpr (LDG) return __ldg(p);
  else return *p;
}
template <typename T, typename S, bool LDG = true>
__device__ __forceinline__ void load_geo(const S* __restrict__ tab, size_t plane, size_t c, Geo<T>& g) {
#pragma unroll
  for (int f = 0; f < 10; f++) g.gcov[f] = (T)tab_ld<LDG>(tab + (size_t)(HARM_G_GCOV + f) * plane + c);
#pragma unroll
  for (int f = 0; f < 10; f++) g.gcon[f] = (T)tab_ld<LDG>(tab + (size_t)(HARM_G_GCON + f) * plane + c);
  g.gcovpert_tt = (T)tab_ld<LDG>(tab + (size_t)HARM_G_GCOVPERT_TT * plane + c);
  g.alpha = (T)tab_ld<LDG>(tab + (size_t)HARM_G_ALPHA * plane + c);
  g.betasqoalphasq = (T)tab_ld<LDG>(tab + (size_t)HARM_G_BETASQOALPHASQ * plane + c);
  g.beta1 = (T)tab_ld<LDG>(tab + (size_t)(HARM_G_BETA + 0) * plane + c);
  g.beta2 = (T)tab_ld<LDG>(tab + (size_t)(HARM_G_BETA + 1) * plane + c);
  g.beta3 = (T)tab_ld<LDG>(tab + (size_t)(HARM_G_BETA + 2) * plane + c);
  g.gdet = (T)tab_ld<LDG>(tab + (size_t)HARM_G_GDET * plane + c);
  g.igdet = (T)tab_ld<LDG>(tab + (size_t)HARM_G_IGDET * plane + c);
}

template <typename T>
struct State {
  T ucon[4], ucov[4], bsq, pressure, plus1ud0, gamma, qsq;
};

template <typename T>
__device__ __forceinline__ void lower(const T* u, const Geo<T>& g, T* d) {
  d[0] = g.gcov[0] * u[0] + g.gcov[1] * u[1] + g.gcov[2] * u[2] + g.gcov[3] * u[3];
  d[1] = g.gcov[1] * u[0] + g.gcov[4] * u[1] + g.gcov[5] * u[2] + g.gcov[6] * u[3];
  d[2] = g.gcov[2] * u[0] + g.gcov[5] * u[1] + g.gcov[7] * u[2];
  d[3] = g.gcov[3] * u[0] + g.gcov[6] * u[1] + g.gcov[9] * u[3];
}
template <typename T>
__device__ __forceinline__ void raise(const T* d, const Geo<T>& g, T* u) {
  u[0] = g.gcon[0] * d[0] + g.gcon[1] * d[1] + g.gcon[2] * d[2] + g.gcon[3] * d[3];
  u[1] = g.gcon[1] * d[0] + g.gcon[4] * d[1] + g.gcon[5] * d[2] + g.gcon[6] * d[3];
  u[2] = g.gcon[2] * d[0] + g.gcon[5] * d[1] + g.gcon[7] * d[2] + g.gcon[8] * d[3];
  u[3] = g.gcon[3] * d[0] + g.gcon[6] * d[1] + g.gcon[8] * d[2] + g.gcon[9] * d[3];
}

template <typename T>
__device__ __forceinline__ T qsq_of(const T* pr, const Geo<T>& g) {
  T u1 = pr[HARM_U1], u2 = pr[HARM_U2], u3 = pr[HARM_U3];
  return g.gcov[4] * u1 * u1 + g.gcov[7] * u2 * u2 + g.gcov[9] * u3 * u3 +
         T(2.) * (g.gcov[5] * u1 * u2 + g.gcov[6] * u1 * u3);
}

template <typename T>
__device__ __forceinline__ void ucon_of(const T* pr, const Geo<T>& g, T* ucon, T& gamma, T& qsq) {
  T q = qsq_of(pr, g);
  q = (q >= T(0)) ? q : T(0);
  qsq = q;
  gamma = sqrt(T(1) + q);
  ucon[0] = gamma / g.alpha;
  ucon[1] = pr[HARM_U1] - ucon[0] * g.beta1;
  ucon[2] = pr[HARM_U2] - ucon[0] * g.beta2;
  ucon[3] = pr[HARM_U3] - ucon[0] * g.beta3;
}

// B^i B_i and B^i u_i
template <typename T>
__device__ __forceinline__ void bdots(const T* pr, const Geo<T>& g, const T* ucov, T* Bcov, T& Bsq, T& udotB) {
  const T B1 = pr[HARM_B1], B2 = pr[HARM_B2], B3 = pr[HARM_B3];
  Bcov[0] = B1 * g.gcov[1] + B2 * g.gcov[2] + B3 * g.gcov[3];
  Bcov[1] = B1 * g.gcov[4] + B2 * g.gcov[5] + B3 * g.gcov[6];
  Bcov[2] = B1 * g.gcov[5] + B2 * g.gcov[7] + B3 * g.gcov[8];
  Bcov[3] = B1 * g.gcov[6] + B2 * g.gcov[8] + B3 * g.gcov[9];
  Bsq = B1 * Bcov[1] + B2 * Bcov[2] + B3 * Bcov[3];
  udotB = B1 * ucov[1] + B2 * ucov[2] + B3 * ucov[3];
}

template <typename T>
__device__ __forceinline__ void get_state(const T* pr, const Geo<T>& g, T gam, State<T>& q) {
  ucon_of(pr, g, q.ucon, q.gamma, q.qsq);
  lower(q.ucon, g, q.ucov);
  T ud0tilde = pr[HARM_U1] * g.gcov[1] + pr[HARM_U2] * g.gcov[2] + pr[HARM_U3] * g.gcov[3];
  T alphasq = g.alpha * g.alpha;
  q.plus1ud0 = ud0tilde + (g.gcovpert_tt - alphasq * (g.betasqoalphasq + q.qsq)) / (T(1) + q.gamma * g.alpha);
  T Bcov[4], Bsq, udotB;
  bdots(pr, g, q.ucov, Bcov, Bsq, udotB);
  q.bsq = (Bsq + udotB * udotB) / (q.ucon[0] * q.ucon[0]);
  q.pressure = (gam - T(1)) * pr[HARM_UU];
}

// Flux in direction dir (0 = conserved variables), times gd (sqrt(-g) for UEVOLVE, 1 for
// geometry-free U).
template <typename T>
__device__ __forceinline__ void primtoflux(const T* pr, const State<T>& q, int dir, const Geo<T>& g, T gd, T* F) {
  const T rho = pr[HARM_RHO], u = pr[HARM_UU], P = q.pressure, w = P + rho + u;
  const T ud = q.ucon[dir];
  T ma[4], em[4];
  ma[0] = (P + u) * ud * q.ucov[0] + rho * ud * q.plus1ud0;
  ma[1] = w * ud * q.ucov[1];
  ma[2] = w * ud * q.ucov[2];
  ma[3] = w * ud * q.ucov[3];
  ma[dir] += P;
  T Bcov[4], Bsq, udotB;
  bdots(pr, g, q.ucov, Bcov, Bsq, udotB);
  const T Bd = (dir == 0) ? T(0) : pr[HARM_B1 + dir - 1];
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
    em[mu] = Bsq * ud * q.ucov[mu] - Bd * Bcov[mu] - udotB * (Bd * q.ucov[mu] + Bcov[mu] * ud);
  em[dir] += T(0.5) * (Bsq + udotB * udotB);
  const T ig2 = T(1) / (q.ucon[0] * q.ucon[0]);
  F[HARM_RHO] = rho * ud * gd;
#pragma unroll
  for (int mu = 0; mu < 4; mu++) F[HARM_UU + mu] = (ma[mu] + em[mu] * ig2) * gd;
  if (dir > 0) {
    F[HARM_B1] = ((pr[HARM_B1] * ud - Bd * q.ucon[1]) / q.ucon[0]) * gd;
    F[HARM_B2] = ((pr[HARM_B2] * ud - Bd * q.ucon[2]) / q.ucon[0]) * gd;
    F[HARM_B3] = ((pr[HARM_B3] * ud - Bd * q.ucon[3]) / q.ucon[0]) * gd;
  } else {
    F[HARM_B1] = pr[HARM_B1] * gd;
    F[HARM_B2] = pr[HARM_B2] * gd;
    F[HARM_B3] = pr[HARM_B3] * gd;
  }
}

template <typename T>
struct Eps;
template <>
struct Eps<double> {
  static constexpr double eps = 2.220446049250313e-16, small = 1e-300;
};
template <>
struct Eps<float> {
  static constexpr float eps = 1.1920929e-07f, small = 1e-35f;
};

// vchar + simplefast (USESASHAREWRITE form of the discriminant)
template <typename T>
__device__ __forceinline__ void vchar(const T* pr, const State<T>& q, int dir, const Geo<T>& g, T gam, T& vmax, T& vmin) {
  T rho = pr[HARM_RHO], u = pr[HARM_UU];
  if (u < T(0)) u = T(0);
  if (rho < T(0)) rho = Eps<T>::small;
  T P = q.pressure, WW = rho + u + P, cs2;
  if (WW > T(0)) {
    T pp = (gam - T(1)) * u, h = rho + u + pp;
    cs2 = gam * pp / h;
  } else {
    WW = cs2 = Eps<T>::small;
  }
  if (cs2 >= T(1)) cs2 = T(1) - Eps<T>::eps * T(10);
  else if (cs2 <= T(0)) cs2 = Eps<T>::small;
  T EF = Eps<T>::small + fabs(q.bsq + WW);
  T va2 = q.bsq / EF;
  T cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < T(0) && cms2 / (cs2 + va2) > -Eps<T>::eps * T(100)) cms2 = T(0);
  if (cms2 > T(1) && (cms2 < T(1) + Eps<T>::eps * T(100) || rho < T(0))) cms2 = T(1);
  const T Asq = g.gcon[sym(dir, dir)], Bsq = g.gcon[0], AB = g.gcon[dir];
  const T Au = q.ucon[dir], Bu = q.ucon[0];
  const T Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  const T B = T(2) * (AuBu * (T(1) - cms2) - AB * cms2);
  const T A = Bu2 * (T(1) - cms2) - Bsq * cms2;
  T discr = T(4) * cms2 * ((AB * AB - Asq * Bsq) * cms2 + (T(2) * AB * Au * Bu - Asq * Bu2 - Bsq * Au2) * (cms2 - T(1)));
  if (discr < T(0)) discr = T(0);
  discr = sqrt(discr);
  const T vm = -(-B + discr) / (T(2) * A), vp = -(-B - discr) / (T(2) * A);
  if (vp < vm) { vmax = vm; vmin = vp; }
  else { vmax = vp; vmin = vm; }
}

// limit_gamma (fixup.c:2723).  Returns true if the velocity was rescaled.
template <typename T>
__device__ __forceinline__ bool limit_gamma(T gammamax, T* pr, const Geo<T>& g) {
  if (gammamax <= T(1)) return false;
  T q = qsq_of(pr, g);
  q = (q >= T(0)) ? q : T(0);
  T gamma = sqrt(T(1) + q);
  if (gamma > gammamax && gamma != T(1)) {
    T pref = (gammamax * gammamax - T(1)) / (gamma * gamma - T(1));
    if (pref < T(0)) return false;
    T f = sqrt(pref);
    pr[HARM_U1] *= f;
    pr[HARM_U2] *= f;
    pr[HARM_U3] *= f;
    return true;
  }
  return false;
}

// MINMOD-limited MC slope (interppoint.c:753-775)
template <typename T>
__device__ __forceinline__ T mc_slope(T yl, T yc, T yr) {
  T Dqm = T(2) * (yc - yl), Dqp = T(2) * (yr - yc), Dqc = T(0.5) * (yr - yl);
  T m1 = (Dqm * Dqp <= T(0)) ? T(0) : ((fabs(Dqm) < fabs(Dqp)) ? Dqm : Dqp);
  return (Dqc * m1 <= T(0)) ? T(0) : ((fabs(Dqc) < fabs(m1)) ? Dqc : m1);
}


// ---------------------------------------------------------------- PPM (para4)
// interppoint.para.c:568-760 with PARA2LIM=MC and the defaults of para_and_paraenohybrid.h;
// checkparamonotonicity :1069.  y points at the cell, uses y[-2..2].
template <typename T>
__device__ __forceinline__ T minmod2(T a, T b) {
  return (a * b <= T(0)) ? T(0) : ((fabs(a) < fabs(b)) ? a : b);
}

// checkparamonotonicity (interppoint.para.c:1069) with smooth = 0, PARAGENDQALLOWEXTREMUM = 0,
// NONMONOLIM = 0 and the a6 coefficient of point values (4)
template <typename T>
__device__ __forceinline__ void para_monotonicity(T y0, T& l, T& r) {
  const T a6 = T(4);
  T qa = (r - y0) * (y0 - l), qd = (r - l), qe = a6 * (y0 - T(0.5) * (l + r));
  if (qa <= T(0)) {
    l = y0;
    r = y0;
  } else {
    if (qd * (qd - qe) < T(0)) l = (-(T(2) + a6) * r + T(2) * a6 * y0) / (a6 - T(2));
    else if (qd * (qd + qe) < T(0)) r = (-(T(2) + a6) * l + T(2) * a6 * y0) / (a6 - T(2));
  }
}

template <typename T>
__device__ __forceinline__ void para4_cell(const T* y, T& lout, T& rout) {
  T dq[3];
#pragma unroll
  for (int mm = -1; mm <= 1; mm++) {
    T dq1m = y[mm] - y[mm - 1], dq1p = y[mm + 1] - y[mm];
    T Dqc = T(0.5) * (y[mm + 1] - y[mm - 1]);
    dq[mm + 1] = minmod2(Dqc, minmod2(T(2) * dq1m, T(2) * dq1p));
  }
  T ddql = dq[1] - dq[0], ddqr = dq[2] - dq[1];
  T l = T(0.5) * (y[0] + y[-1]) - ddql * T(1.0 / 8.0);
  T r = T(0.5) * (y[1] + y[0]) - ddqr * T(1.0 / 8.0);
  para_monotonicity<T>(y[0], l, r);
  lout = l;
  rout = r;
}

// ---------------------------------------------------------------- line PPM (PARALINE)
// pass_1d_line_multipl_paraline (interpline.para.c:8) with DOPPMREDUCE=1 and the other
// switches of para_and_paraenohybrid.h at their defaults: MC slopes that keep the extremum
// (get_limit_slopes_paraline :165, PARALINE2EXTREME=1), continuous face values (paracont
// interppoint.para.c:958), both edges pulled towards the cell value by the flattening
// coefficient Fi (paraflatten :1305), then checkparamonotonicity (:1069).  Fi is FLASH's
// flattener (Ficalc :1356, ftilde :1316, SP0 = 0.75) of V = sqrt(-g) rho u^dir and the total
// pressure P = p + b^2/2 of the cells -3..3 (get_V_and_P interpline.c:2964).  The reference's
// max/min (phys.tools.c:2356) are a > b ? a : b and a > b ? b : a, kept as written.
template <typename T>
struct ParalineConst;
template <>
struct ParalineConst<double> {
  static constexpr double small = 1.e-300;               // SMALL of a double build
  static constexpr double third = 0x1.5555555555556p-2;  // least double >= the long double 1/3
};
template <>
struct ParalineConst<float> {
  static constexpr float small = 1.e-35f;                // SMALL of a float build
  static constexpr float third = 0x1.555556p-2f;         // least float >= 1/3
};

// ftilde of one cell from V at its neighbours -1, +1 and P at -2..2
template <typename T>
__device__ __forceinline__ T paraline_ftilde(T vm1, T vp1, T pm2, T pm1, T pp1, T pp2) {
  using K = ParalineConst<T>;
  const T P2diff = pp2 - pm2;
  const T Pbottom = copysign(T(1), P2diff) / (fabs(P2diff) + K::small);
  const T Sp = (pp1 - pm1) * Pbottom;
  const T m = T(10) * (Sp - T(0.75));
  const T mn = (T(1) > m) ? m : T(1);
  T Ft = (T(0) > mn) ? T(0) : mn;
  const T a = fabs(pp1), b = fabs(pm1);
  const T Ft1 = fabs(pp1 - pm1) / (((a > b) ? b : a) + K::small);
  Ft *= (Ft1 >= K::third) ? T(1) : T(0);
  Ft *= (vp1 - vm1 <= T(0)) ? T(1) : T(0);
  return Ft;
}

// Fi of the cell at v[3], p[3] (v, p: cells -3..3): the larger of its own ftilde and that of
// its neighbour on the side of lower pressure (shift -sign(P[1] - P[-1]), ties to +1)
template <typename T>
__device__ __forceinline__ T paraline_fi(const T* v, const T* p) {
  const T f0 = paraline_ftilde<T>(v[2], v[4], p[1], p[2], p[4], p[5]);
  const T f1 = (p[4] - p[2] > T(0)) ? paraline_ftilde<T>(v[1], v[3], p[0], p[1], p[3], p[4])
                                    : paraline_ftilde<T>(v[3], v[5], p[2], p[3], p[5], p[6]);
  return (f0 > f1) ? f0 : f1;
}

template <typename T>
__device__ __forceinline__ T paraline_dq(T ym, T y0, T yp) {
  const T Dqm = T(2) * (y0 - ym), Dqp = T(2) * (yp - y0), Dqc = T(0.5) * (yp - ym);
  const T m1 = (fabs(Dqm) < fabs(Dqp)) ? Dqm : Dqp;
  return (fabs(Dqc) < fabs(m1)) ? Dqc : m1;
}

// edges of the cell at y[0] (uses y[-2..2]) with flattening coefficient fi
template <typename T>
__device__ __forceinline__ void paraline_cell(const T* y, T fi, T& lout, T& rout) {
  const T dqm = paraline_dq<T>(y[-2], y[-1], y[0]), dq0 = paraline_dq<T>(y[-1], y[0], y[1]);
  const T dqp = paraline_dq<T>(y[0], y[1], y[2]);
  T l = T(0.5) * (y[0] + y[-1]) - (dq0 - dqm) * T(1.0 / 8.0);
  T r = T(0.5) * (y[1] + y[0]) - (dqp - dq0) * T(1.0 / 8.0);
  l = fi * y[0] + (T(1) - fi) * l;
  r = fi * y[0] + (T(1) - fi) * r;
  para_monotonicity<T>(y[0], l, r);
  lout = l;
  rout = r;
}

// ---------------------------------------------------------------- WENO5 (WENO5BND)
// eno_line_reconstruct reconstructeno.c:333 for CVT_C2E: smoothness indicators
// (compute_cf_stencil_weights :1693), desensitising and normalisation (:2001, :2292),
// 1/(beta+eps)^2 weights (:2211), limit_weight (:3015), optimal face weights (:1905),
// WENO3 lower-order weights, weight-ratio stencil reduction (compute_weights_ratios :2311,
// choose_weno_order :2442) raised by the momentum-flux jump of the cell
// (apply_additional_reduction_to_weights :795, dP of compute_df_line_new interpline.c:3557),
// edge values (eno_cvt :884), and the SMONO monotonicity indicator of the 5-point polynomial
// (compute_mono_indicator_point_eno5 interpline.smono.c:517): a monotone cell (indicator 1)
// takes the 5-point edge values, a partly monotone one blends its WENO5 weights and its
// output towards them (mono_adjust_unoptimized_weights reconstructeno.c:852).  Sums use the
// symmetric pairwise order of get_sum_of_elements.
// eps: WENO_EPSILON = (500 DBL_EPSILON)^2 (desensitising and weight ratios), the same value
// in both arithmetic types so that the FP32 reconstruction is the FP64 algorithm up to
// rounding; weps: the epsilon of 1/(beta+eps)^2, which in FP32 is raised to 1e-18 so that its
// square stays a normal number (it only acts where a normalised beta is below ~1e-18, far
// under FP32 resolution); tiny: the smallest normal number (divisions by zero sums).
// smono: SMONO_EPSILON = 500 DBL_EPSILON in both types: the FP32 indicator then switches
// where the FP64 one does, up to the FP32 rounding of derivatives that are already within
// ~1e-7 of the stencil's magnitude (data that flat give the same edges either way); small:
// the reference's SMALL of the type (global.depnmemonics.h:488-493), the guard of the dP
// denominator.
template <typename T>
struct WenoEps;
template <>
struct WenoEps<double> {
  static constexpr double eps = (500.0 * 2.220446049250313e-16) * (500.0 * 2.220446049250313e-16);
  static constexpr double weps = eps;
  static constexpr double tiny = 2.2250738585072014e-308;  // DBL_MIN
  static constexpr double smono = 500.0 * 2.220446049250313e-16;
  static constexpr double small = 1.e-300;
};
template <>
struct WenoEps<float> {
  static constexpr float eps = (float)((500.0 * 2.220446049250313e-16) * (500.0 * 2.220446049250313e-16));
  static constexpr float weps = 1e-18f;
  static constexpr float tiny = 1.17549435e-38f;  // FLT_MIN
  static constexpr float smono = (float)(500.0 * 2.220446049250313e-16);
  static constexpr float small = 1.e-35f;
};

template <typename T>
__device__ __forceinline__ T symsum3(T a0, T a1, T a2) {
  T s = T(0);
  s += a0 + a2;
  s += a1 * T(1);
  return s;
}
template <typename T>
__device__ __forceinline__ T symsum2(T a0, T a1) {
  T s = T(0);
  s += a0 + a1;
  s += a1 * T(0);  // the loop's next element, multiplied by (count odd) = 0
  return s;
}

// Division inside the WENO weights.  FP64: IEEE division (the oracle's operations).  FP32
// (mixed path): the fast reciprocal-multiply form, error of 2 ulp; the weights only steer the
// stencil combination, so this stays far inside the FP32 reconstruction's own rounding.
template <typename T>
__device__ __forceinline__ T wdiv(T a, T b) {
  return a / b;
}
template <>
__device__ __forceinline__ float wdiv<float>(float a, float b) {
  return __fdividef(a, b);
}

// Division by a compile-time constant: FP64 divides; FP32 multiplies by the folded reciprocal.
template <typename T>
__device__ __forceinline__ T wdivk(T a, T b) {
  return a / b;
}
template <>
__device__ __forceinline__ float wdivk<float>(float a, float b) {
  return a * (1.0f / b);
}

// Several values over one denominator: FP64 divides each (the oracle's operations); FP32
// multiplies by one fast reciprocal.
template <typename T>
struct WScale {
  T d;
  __device__ __forceinline__ explicit WScale(T den) : d(den) {}
  __device__ __forceinline__ T operator()(T a) const { return a / d; }
};
template <>
struct WScale<float> {
  float r;
  __device__ __forceinline__ explicit WScale(float den) {
#ifdef __CUDA_ARCH__
    r = __fdividef(1.0f, den);
#else
    r = 1.0f / den;  // host pass only parses this; the kernels use the line above
#endif
  }
  __device__ __forceinline__ float operator()(float a) const { return a * r; }
};

template <typename T>
__device__ __forceinline__ T limit_weight(int order, T w) {
  const T avg = T(1) / T(order), w1 = T(0.2) * avg, w2 = (T(1) - T(0.2)) * avg, w3 = (T(1) + T(0.2)) * avg, w4 = T(1);
  if constexpr (sizeof(T) == 4) {
    // FP32: the limiter is continuous and piecewise linear, 0 | ramp to avg | avg | ramp to 1,
    // so it is the lower ramp clamped to [0, avg] plus the part of the upper ramp above avg:
    // min/max instead of compares and selects, no divergent branches (the same values away
    // from the break points, within a rounding at them)
    const T lo = wdivk<T>(avg * (w - w1), w2 - w1);
    const T up = wdivk<T>((w - w3) * (w4 - avg), w4 - w3);
    return fmaxf(fminf(lo, avg), T(0)) + fmaxf(up, T(0));
  } else {
    if (w < w1) return T(0);
    if (w < w2) return wdivk<T>(avg * (w - w1), w2 - w1);
    if (w < w3) return avg;
    return wdivk<T>((w - w3) * (w4 - avg), w4 - w3) + avg;
  }
}

// unoptimised (limited, normalised) weights of the three 3-point stencils of the cell at u
template <typename T>
__device__ __forceinline__ void weno5_unopt(const T* u, T* w) {
  T fd0 = -(T(3) * u[0] + u[2]) + T(4) * u[1];
  T fd1 = u[1] - u[-1];
  T fd2 = (T(3) * u[0] + u[-2]) - T(4) * u[-1];
  T sd0 = (u[0] + u[2]) - T(2) * u[1];
  T sd1 = (u[-1] + u[1]) - T(2) * u[0];
  T sd2 = (u[0] + u[-2]) - T(2) * u[-1];
  T b[3];
  b[0] = T(13. / 12.) * sd0 * sd0 + T(1. / 4.) * fd0 * fd0;
  b[1] = T(13. / 12.) * sd1 * sd1 + T(1. / 4.) * fd1 * fd1;
  b[2] = T(13. / 12.) * sd2 * sd2 + T(1. / 4.) * fd2 * fd2;
  // desensitise: sum of u^2 over the 5 cells in the symmetric order
  T normu = T(0);
  normu += u[-2] * u[-2] + u[2] * u[2];
  normu += u[-1] * u[-1] + u[1] * u[1];
  normu += u[0] * u[0] * T(1);
  const T ee = normu * WenoEps<T>::eps;
#pragma unroll
  for (int s = 0; s < 3; s++) b[s] += ee;
  T sb = symsum3(b[0], b[1], b[2]);
  const WScale<T> nb(sb + WenoEps<T>::tiny);
#pragma unroll
  for (int s = 0; s < 3; s++) b[s] = nb(b[s]);
#pragma unroll
  for (int s = 0; s < 3; s++) {
    T t = b[s] + WenoEps<T>::weps;
    t *= t;
    w[s] = wdiv<T>(T(1), t);
  }
  T sw = symsum3(w[0], w[1], w[2]);
  const WScale<T> n1(sw + T(0));
#pragma unroll
  for (int s = 0; s < 3; s++) w[s] = n1(w[s]);
#pragma unroll
  for (int s = 0; s < 3; s++) w[s] = limit_weight<T>(3, w[s]);
  sw = symsum3(w[0], w[1], w[2]);
  const WScale<T> n2(sw + T(0));
#pragma unroll
  for (int s = 0; s < 3; s++) w[s] = n2(w[s]);
}

// the same for the two 2-point stencils (WENO3)
template <typename T>
__device__ __forceinline__ void weno3_unopt(const T* u, T* w) {
  T fd0 = u[1] - u[0], fd1 = u[0] - u[-1];
  T b[2] = {fd0 * fd0, fd1 * fd1};
  T normu = T(0);
  normu += u[-1] * u[-1] + u[1] * u[1];
  normu += u[0] * u[0] * T(1);
  const T ee = normu * WenoEps<T>::eps;
  b[0] += ee;
  b[1] += ee;
  T sb = symsum2(b[0], b[1]);
  const WScale<T> nb(sb + WenoEps<T>::tiny);
  b[0] = nb(b[0]);
  b[1] = nb(b[1]);
#pragma unroll
  for (int s = 0; s < 2; s++) {
    T t = b[s] + WenoEps<T>::weps;
    t *= t;
    w[s] = wdiv<T>(T(1), t);
  }
  T sw = symsum2(w[0], w[1]);
  const WScale<T> n1(sw + T(0));
  w[0] = n1(w[0]);
  w[1] = n1(w[1]);
  w[0] = limit_weight<T>(2, w[0]);
  w[1] = limit_weight<T>(2, w[1]);
  sw = symsum2(w[0], w[1]);
  const WScale<T> n2(sw + T(0));
  w[0] = n2(w[0]);
  w[1] = n2(w[1]);
}

// SMONO indicator of the cell at y (y[-2..2]): the left and right edge derivatives of orders
// 1..3 of the 5-point polynomial (order 1 also min-modded with the outer one-sided difference)
// must agree in sign; the smallest of them against 500 epsilons of the stencil's magnitude
// gives 0 .. 1 (SMONO_DO_SMOOTH_TRANSITION)
template <typename T>
__device__ __forceinline__ T smono_indicator(const T* y) {
  const T k12 = T(12), k2 = T(2);
  T ld1 = wdivk<T>(((T(-3) * y[-2] + y[2]) + (T(-10) * y[-1] - T(6) * y[1])) + T(18) * y[0], k12);
  T ld2 = wdivk<T>(((T(11) * y[-2] - y[2]) + (T(-20) * y[-1] + T(4) * y[1])) + T(6) * y[0], k12);
  T ld3 = wdivk<T>(((T(-3) * y[-2] - y[2]) + (T(10) * y[-1] + T(6) * y[1])) - T(12) * y[0], k2);
  T rd1 = wdivk<T>(((-y[-2] + T(3) * y[2]) + (T(6) * y[-1] + T(10) * y[1])) - T(18) * y[0], k12);
  T rd2 = wdivk<T>(((-y[-2] + T(11) * y[2]) + (T(4) * y[-1] - T(20) * y[1])) + T(6) * y[0], k12);
  T rd3 = wdivk<T>(((y[-2] + T(3) * y[2]) - (T(6) * y[-1] + T(10) * y[1])) + T(12) * y[0], k2);
  auto mm = [](T a, T b) -> T { return (a * b <= T(0)) ? T(0) : ((fabs(a) < fabs(b)) ? a : b); };
  ld1 = mm(ld1, y[-1] - y[-2]);
  rd1 = mm(rd1, y[2] - y[1]);
  T minabs = T(sizeof(T) == 8 ? 1.e+100 : 1.e+30);
  const T m1 = fabs(mm(ld1, rd1)), m2 = fabs(mm(ld2, rd2)), m3 = fabs(mm(ld3, rd3));
  minabs = (minabs < m1) ? minabs : m1;
  minabs = (minabs < m2) ? minabs : m2;
  minabs = (minabs < m3) ? minabs : m3;
  const T norm = fabs(y[0]) + ((fabs(y[-1]) + fabs(y[1])) + (fabs(y[-2]) + fabs(y[2])));
  const T cutoff = norm * WenoEps<T>::smono + WenoEps<T>::tiny;
  T v = wdiv<T>(minabs - T(0), cutoff - T(0));
  v = (T(1) < v) ? T(1) : v;
  return (T(0) > v) ? T(0) : v;
}

// the cell's WENO5 weights as the ratios and the edges use them: equal weights where the
// cell is monotone (m = 1), the unoptimised weights blended towards equal ones by m
template <typename T>
__device__ __forceinline__ void weno5_cell_weights(const T* u, T m, T* w) {
  if (m == T(1)) {
    w[0] = w[1] = w[2] = T(1) / T(3);
    return;
  }
  weno5_unopt<T>(u, w);
  if (m > T(0) && m < T(1)) {
#pragma unroll
    for (int s = 0; s < 3; s++) w[s] = (T(1) - m) * w[s] + m * (T(1) / T(3));
  }
}

// lower-order fraction of a cell from the ratios of its outer weights to its neighbours' (at
// distance 2) inner ones
template <typename T>
__device__ __forceinline__ T weno_frac(const T* w, const T* wm, const T* wp) {
  const T E = WenoEps<T>::eps;
  T rl = wdiv<T>(w[2] + E, wm[0] + E);
  T rr = wdiv<T>(w[0] + E, wp[2] + E);
  T ratio = fmin(rl, rr);
  T f = wdivk<T>(ratio - T(1.3), T(1.6) - T(1.3));
  return fmax(T(0), fmin(f, T(1)));
}

// the strength of the dP reduction of a cell: min((|dP| - 0.25)/0.25, 1), at most 0 where
// |dP| <= 0.25 (REDUCE_DP_FRACTION = 0.5); the cell's fraction is then raised to its
// neighbours' scaled by it
template <typename T>
__device__ __forceinline__ T weno_dp_strength(T dP) {
  T ss = wdivk<T>(fabs(dP) - T(0.5) * T(0.5), T(0.5) * T(0.5));
  return (ss < T(1)) ? ss : T(1);
}
template <typename T>
__device__ __forceinline__ T weno_lof(T f, T fm, T fp, T ss) {
  T t = ss * fp;
  T l = (f > t) ? f : t;
  t = ss * fm;
  return (l > t) ? l : t;
}

// the line quantities of one cell for dP (compute_df_line_new): par = |(1 + u_t) u^dir|,
// veff = sign(sqrt(-g) rho u^dir) par / (sqrt(par) + SMALL),
// upar = |(u + p + b^2)(|u^dir| u_t) + p + b^2/2 - b^dir b_t|
template <typename T>
__device__ __forceinline__ void weno_dp_of_state(const T* pr, const Geo<T>& g, const State<T>& q, int dir, T& par,
                                                 T& veff, T& upar) {
  T bcon[4], bcov0;
  bcon[0] = pr[HARM_B1] * q.ucov[1] + pr[HARM_B2] * q.ucov[2] + pr[HARM_B3] * q.ucov[3];
#pragma unroll
  for (int j = 1; j <= 3; j++) bcon[j] = (pr[HARM_B1 - 1 + j] + bcon[0] * q.ucon[j]) / q.ucon[0];
  bcov0 = g.gcov[0] * bcon[0] + g.gcov[1] * bcon[1] + g.gcov[2] * bcon[2] + g.gcov[3] * bcon[3];
  const T ud = q.ucon[dir];
  const T V = g.gdet * pr[HARM_RHO] * ud;
  const T btt = -bcon[dir] * bcov0;
  const T ptot = q.pressure + T(0.5) * q.bsq;
  par = fabs(q.plus1ud0 * ud);
  veff = copysign(T(1), V) * par / (sqrt(par) + WenoEps<T>::small);
  upar = fabs((pr[HARM_UU] + q.pressure + q.bsq) * (fabs(ud) * q.ucov[0]) + ptot + btt);
}
template <typename T>
__device__ __forceinline__ void weno_dp_cell(const T* pr, const Geo<T>& g, T gam, int dir, T& par, T& veff, T& upar) {
  State<T> q;
  get_state<T>(pr, g, gam, q);
  weno_dp_of_state<T>(pr, g, q, dir, par, veff, upar);
}
// dP of a cell from its rho, par, upar and its neighbours' veff, upar
template <typename T>
__device__ __forceinline__ T weno_dp(T rho, T par, T upar, T veffm, T veffp, T uparm, T uparp) {
  const T dv = veffp - veffm;
  return (fabs(rho * dv * dv) + fabs(uparp - uparm)) / (fabs(rho * par) + fabs(upar) + WenoEps<T>::small);
}

// the 5-point edge values (c2e_simple_eno reconstructeno.c:984)
template <typename T>
__device__ __forceinline__ T weno_edge5(const T* u, bool right) {
  const T c0 = right ? T(3. / 128.) : T(-5. / 128.), c1 = right ? T(-5. / 32.) : T(15. / 32.), c2 = T(45. / 64.),
          c3 = right ? T(15. / 32.) : T(-5. / 32.), c4 = right ? T(-5. / 128.) : T(3. / 128.);
  T s = T(0);
  s += c0 * u[-2] + c4 * u[2];
  s += c1 * u[-1] + c3 * u[1];
  s += c2 * u[0] * T(1);
  return s;
}

// left and right edge values of the cell at u from its (mono-adjusted) WENO5 weights w, its
// final lower-order fraction f and its SMONO indicator m
template <typename T>
__device__ __forceinline__ void weno5_edges(const T* u, const T* w, T f, T m, T& yl, T& yr) {
  T y5l = T(0), y5r = T(0);
  if (m != T(0)) {
    y5l = weno_edge5<T>(u, false);
    y5r = weno_edge5<T>(u, true);
  }
  if (m >= T(1)) {
    yl = y5l;
    yr = y5r;
    return;
  }
  // optimal face weights (order 3)
  T wl[3] = {w[0] * T(1. / 16.), w[1] * T(5. / 8.), w[2] * T(5. / 16.)};
  T wr[3] = {w[0] * T(5. / 16.), w[1] * T(5. / 8.), w[2] * T(1. / 16.)};
  T sl = symsum3(wl[0], wl[1], wl[2]), sr = symsum3(wr[0], wr[1], wr[2]);
  const WScale<T> nl(sl + WenoEps<T>::tiny), nr(sr + WenoEps<T>::tiny);
#pragma unroll
  for (int s = 0; s < 3; s++) {
    wl[s] = nl(wl[s]);
    wr[s] = nr(wr[s]);
  }
  const bool two = (T(0) < f);
  if (two) {
#pragma unroll
    for (int s = 0; s < 3; s++) {
      wl[s] *= (T(1) - f);
      wr[s] *= (T(1) - f);
    }
  }
  // stencil polynomials (c2l/c2r_array3)
  T recl0 = symsum3(T(15. / 8.) * u[0], T(-5. / 4.) * u[1], T(3. / 8.) * u[2]);
  T recl1 = symsum3(T(3. / 8.) * u[-1], T(3. / 4.) * u[0], T(-1. / 8.) * u[1]);
  T recl2 = symsum3(T(-1. / 8.) * u[-2], T(3. / 4.) * u[-1], T(3. / 8.) * u[0]);
  T recr0 = symsum3(T(3. / 8.) * u[0], T(3. / 4.) * u[1], T(-1. / 8.) * u[2]);
  T recr1 = symsum3(T(-1. / 8.) * u[-1], T(3. / 4.) * u[0], T(3. / 8.) * u[1]);
  T recr2 = symsum3(T(3. / 8.) * u[-2], T(-5. / 4.) * u[-1], T(15. / 8.) * u[0]);
  T ul0 = (wl[0] != T(0)) ? wl[0] * recl0 : T(0);
  T ul1 = (wl[1] != T(0)) ? wl[1] * recl1 : T(0);
  T ul2 = (wl[2] != T(0)) ? wl[2] * recl2 : T(0);
  T ur0 = (wr[0] != T(0)) ? wr[0] * recr0 : T(0);
  T ur1 = (wr[1] != T(0)) ? wr[1] * recr1 : T(0);
  T ur2 = (wr[2] != T(0)) ? wr[2] * recr2 : T(0);
  T outl = T(0), outr = T(0);
  outl += symsum3(ul0, ul1, ul2);
  outr += symsum3(ur0, ur1, ur2);
  if (two) {
    T w3[2];
    weno3_unopt<T>(u, w3);
    T l3[2] = {w3[0] * T(1. / 4.), w3[1] * T(3. / 4.)};
    T r3[2] = {w3[0] * T(3. / 4.), w3[1] * T(1. / 4.)};
    T sl3 = symsum2(l3[0], l3[1]), sr3 = symsum2(r3[0], r3[1]);
    const WScale<T> nl3(sl3 + WenoEps<T>::tiny), nr3(sr3 + WenoEps<T>::tiny);
#pragma unroll
    for (int s = 0; s < 2; s++) {
      l3[s] = nl3(l3[s]);
      r3[s] = nr3(r3[s]);
      l3[s] *= f;
      r3[s] *= f;
    }
    T rl0 = symsum2(T(3. / 2.) * u[0], T(-1. / 2.) * u[1]);
    T rl1 = symsum2(T(1. / 2.) * u[-1], T(1. / 2.) * u[0]);
    T rr0 = symsum2(T(1. / 2.) * u[0], T(1. / 2.) * u[1]);
    T rr1 = symsum2(T(-1. / 2.) * u[-1], T(3. / 2.) * u[0]);
    T a0 = (l3[0] != T(0)) ? l3[0] * rl0 : T(0);
    T a1 = (l3[1] != T(0)) ? l3[1] * rl1 : T(0);
    T b0 = (r3[0] != T(0)) ? r3[0] * rr0 : T(0);
    T b1 = (r3[1] != T(0)) ? r3[1] * rr1 : T(0);
    outl += symsum2(a0, a1);
    outr += symsum2(b0, b1);
  }
  yl = (T(1) - m) * outl + m * y5l;
  yr = (T(1) - m) * outr + m * y5r;
}

}  // namespace hb
