// harm_invert.cuh -- FP64 device inversion U -> P (Utoprimgen, utoprimgen.c:32) with
// Jon's 1-D Newton method on E'(W') (utoprim_jon.c:136-1700, 2953-3100, 3665-4330) and
// the HOT2COLD fallback on P^2(W') (trycoldinversion utoprimgen.c:594).
//
// Per cell the work is: the setup scalars {D, B^2, (Q.B)^2, Qt^2, Q.n'} from U and the
// metric (compute_setup_quantities :716), the initial W' (set_guess_Wp :890, or the
// learned guess), at most 200 Newton steps with damping after 10 (general_newton_raphson
// :3853, PRECISEINVERSION tolerances u2p_defs.h:37-48), and W' -> primitives (Wp2prim
// :1346).  Every loop is bounded; nothing here waits on other threads.
#pragma once
#include "harm_device.cuh"

namespace hb {

struct InvC {
  double Bsq, QdotB, QdotBsq, Qtsq, Qdotnp, D;
  double w0, w1, w2;  // wglobal[0..2]
  double gam, gsq_too_big, utsq_too_big;
  int cold;
};

constexpr double kNEWT_TOL = 1E3 * 2.220446049250313e-16;
constexpr double kNEWT_TOL_UR = 2.220446049250313e-16;
constexpr double kMIN_NEWT_TOL = 1E-6;
constexpr int kMAX_NEWT_ITER = 200;
constexpr int kITERDAMPSTART = 10;
constexpr double kVERYBIG = 1.e150;
constexpr double kKINDASMALL = 1.e-100;
constexpr double kBIG = 1.e100;
constexpr double kSQRTMIN = 1.4916681462400413e-154;
constexpr double kSMALL = 1e-300;

// Division inside the Newton iteration.  By default IEEE FP64 division (the operations of the
// C restatement, so the FP64 path matches it to round-off).  A translation unit that defines
// HARM_INVERT_FAST_DIV before including this header (the mixed-precision path) gets the
// reciprocal from the hardware FP64 approximation refined by two Newton-Raphson steps
// (r <- r + r (1 - b r), quadratic convergence from the approximation's relative error), a
// multiply, and reciprocals shared between the divisions of one residual evaluation: within
// an ulp or two of the IEEE quotients for normal operands, with fewer FP64 instructions.
#ifdef HARM_INVERT_FAST_DIV
constexpr bool kFastDiv = true;
__device__ __forceinline__ double frcp(double b) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
  double e = fma(-b, r, 1.0);
  r = fma(r, e, r);
  e = fma(-b, r, 1.0);
  return fma(r, e, r);
}
__device__ __forceinline__ double fdiv(double a, double b) { return a * frcp(b); }
#else
constexpr bool kFastDiv = false;
__device__ __forceinline__ double frcp(double b) { return 1.0 / b; }
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
#endif

__device__ __forceinline__ double utsq_calc(double W, const InvC& c) {
  double SoW = fdiv(c.QdotB, W);
  double top = c.Qtsq + (c.Bsq + 2.0 * W) * SoW * SoW;
  double bot = (c.Bsq * c.Bsq - c.Qtsq) + 2.0 * c.Bsq * W + W * W - SoW * SoW * (c.Bsq + 2.0 * W);
  return fdiv(top, bot);
}
__device__ __forceinline__ bool vsqgtr1(double W, const InvC& c) {
  return W * W * W * (W + 2. * c.Bsq) - c.QdotBsq * (2. * W + c.Bsq) <= W * W * (c.Qtsq - c.Bsq * c.Bsq);
}
__device__ __forceinline__ bool coldgrhd(double Qtsq, double D, double& Wp) {
  double det = D * D + Qtsq;
  if (det < 0.0) return false;
  Wp = (D > 0.0) ? Qtsq / (D + sqrt(det)) : Qtsq / (D - sqrt(det));
  return true;
}

// residual, derivative and Newton step of the hot (E') or cold (P^2) equation
__device__ __forceinline__ void inv_func(double Wp, const InvC& c, double& resid, double& jac, double& dx, double& f) {
  if (kFastDiv && !c.cold) {
    // the same residual and derivative with the divisors' reciprocals formed once
    const double W = Wp + c.D, iW = frcp(W), X = c.Bsq + W + kSMALL, iX = frcp(X), iX2 = iX * iX, iX3 = iX2 * iX;
    const double utsq = utsq_calc(W, c);
    const double gammasq = 1.0 + utsq, gamma = sqrt(gammasq), igsq = frcp(gammasq);
    const double wmrho0 = (Wp - c.D * utsq * frcp(1.0 + gamma)) * igsq;
    if (utsq < -0.9 * c.utsq_too_big || utsq != utsq) {
      resid = -kVERYBIG; jac = 0.0; dx = kVERYBIG; f = 0.5 * resid * resid;
      return;
    }
    const double gm1 = c.gam - 1.0, dpdchi = gm1 / c.gam;
    const double pofchi = dpdchi * wmrho0;
    const double BQ = c.Bsq * c.Qtsq - c.QdotBsq;
    double Ep = c.Qdotnp + Wp - pofchi + 0.5 * c.Bsq + 0.5 * BQ * iX2;
    if (pofchi != pofchi || Ep != Ep) Ep = -kVERYBIG;
    const double Xd = c.Bsq + W, iW3 = iW * iW * iW, iXd = frcp(Xd), iXd3 = iXd * iXd * iXd;
    const double dvsq = -2.0 * iXd3 * (c.Qtsq + c.QdotBsq * (3.0 * W * Xd + c.Bsq * c.Bsq) * iW3);
    const double dwmrho0dvsq = (c.D * (gamma * 0.5 - 1.0) - Wp), drho0dvsq = -c.D * gamma * 0.5;
    const double dpdW = igsq * dpdchi;
    const double dpdvsq = drho0dvsq * 0.0 + dwmrho0dvsq * dpdchi;
    const double dpdWp = dpdW + dpdvsq * dvsq;
    double dE = (1.0 - dpdWp) - BQ * iX3;
    if (dvsq != dvsq || dpdW != dpdW || dpdvsq != dpdvsq || dpdWp != dpdWp || dE != dE) dE = 0.0;
    resid = Ep; jac = dE; dx = -Ep * frcp(dE); f = 0.5 * Ep * Ep;
    return;
  }
  if (!c.cold) {
    double W = Wp + c.D, X = c.Bsq + W + kSMALL, X2 = X * X, X3 = X2 * X;
    double utsq = utsq_calc(W, c);
    double gammasq = 1.0 + utsq, gamma = sqrt(gammasq);
    double wmrho0 = (Wp - c.D * utsq / (1.0 + gamma)) / gammasq;
    if (utsq < -0.9 * c.utsq_too_big || utsq != utsq) {
      resid = -kVERYBIG; jac = 0.0; dx = kVERYBIG; f = 0.5 * resid * resid;
      return;
    }
    double gm1 = c.gam - 1.0, dpdchi = gm1 / c.gam;
    double pofchi = (gm1 / c.gam) * wmrho0;
    double Ep = c.Qdotnp + Wp - pofchi + 0.5 * c.Bsq + 0.5 * (c.Bsq * c.Qtsq - c.QdotBsq) / X2;
    if (pofchi != pofchi || Ep != Ep) Ep = -kVERYBIG;
    double Xd = c.Bsq + W, W3 = W * W * W, Xd3 = Xd * Xd * Xd;
    double dvsq = -2.0 / Xd3 * (c.Qtsq + c.QdotBsq * (3.0 * W * Xd + c.Bsq * c.Bsq) / W3);
    double dwmrho0dW = 1.0 / gammasq;
    double dwmrho0dvsq = (c.D * (gamma * 0.5 - 1.0) - Wp), drho0dvsq = -c.D * gamma * 0.5;
    double dpdW = 0.0 * 0.0 + dwmrho0dW * dpdchi;
    double dpdvsq = drho0dvsq * 0.0 + dwmrho0dvsq * dpdchi;
    double dpdWp = dpdW + dpdvsq * dvsq;
    double dE = (1.0 - dpdWp) - (c.Bsq * c.Qtsq - c.QdotBsq) / X3;
    if (dvsq != dvsq || dpdW != dpdW || dpdvsq != dpdvsq || dpdWp != dpdWp || dE != dE) dE = 0.0;
    resid = Ep; jac = dE; dx = -Ep / dE; f = 0.5 * Ep * Ep;
  } else {
    double W = Wp + c.D, Y = c.Bsq + 2.0 * W, W2 = W * W, S = c.QdotB, D = c.D, Bsq = c.Bsq;
    double r = -c.Qtsq * W2 + Wp * (D + W) * (W2 + Bsq * Y) - Y * S * S;
    double d = 2.0 * (D * ((Bsq + D) * (Bsq + D) - c.Qtsq) - (S * S) + ((Bsq + D) * (Bsq + 5.0 * D) - c.Qtsq) * Wp +
                      3.0 * (Bsq + 2.0 * D) * (Wp * Wp) + 2.0 * (Wp * Wp * Wp));
    resid = r; jac = d; dx = -r / d; f = 0.5 * r * r;
  }
}

__device__ __forceinline__ void validate_Wp(double Wpold, double& Wpnew, const InvC& c) {
  if (Wpnew < -c.D && c.D > 0.0) {
    double Wp = Wpnew / 10.0;
    coldgrhd(c.Qtsq, c.D, Wp);
    Wpnew = Wp * 10.0;
  }
  Wpnew = (fabs(fdiv(Wpnew, c.w1)) > c.gsq_too_big) ? 0.5 * (Wpold + Wpnew) : Wpnew;
}

__device__ __forceinline__ bool ultrarel(double x0, const InvC& c) {
  return (fabs(c.w1) > c.w2) || (fabs(x0) > c.w2);
}
__device__ __forceinline__ bool errcheck(double errx, double x0, const InvC& c) {
  return ultrarel(x0, c) ? (fabs(errx) <= kNEWT_TOL_UR) : (fabs(errx) <= kNEWT_TOL);
}
__device__ __forceinline__ int extracheck(double x0, const InvC& c) { return ultrarel(x0, c) ? 4 : 2; }

// general_newton_raphson, n=1, no line search.  Returns 0/1 (retval), updates flag.
// GATED: when the first Newton step from the start is larger than `gate` relative to
// max(|w0|, |x|) (the scale of the convergence test), the start is judged poor and the
// iteration stops there, returning 2 with xio unchanged (one iteration counted).
template <bool GATED = false>
static __device__ int newton(int8_t& flag, double& xio, const InvC& c, int& lntries, int& nstroke, double gate = 0.0) {
  double x = xio, x_old = x, x_older = x;
  double dx, dx_old = kVERYBIG, resid, jac, f = 1.0, errx = 1.0, damp = 1.0;
  int n_iter = 0, diddamp = 0, i_extra = 0, doing_extra = 0;
  bool keep = true;
  while (keep) {
    nstroke++;
    lntries++;
    if (lntries > kITERDAMPSTART && diddamp == 0) damp = 0.5;
    inv_func(x, c, resid, jac, dx, f);
    if (GATED && n_iter == 0) {
      const double first = (c.w0 == 0.) ? fabs(dx) : fabs(dx) / fmax(fabs(c.w0), fabs(x));
      if (!(first <= gate)) return 2;
    }
    x_older = x_old;
    x_old = x;
    diddamp = 0;
    if (n_iter == 0) {
      x_older = x; x_old = x; dx_old = dx;
    } else {
      if (resid <= -kVERYBIG || jac == 0.0) {
        damp = 0.5 * damp;
        x = x_older;
        dx = dx_old;
        diddamp = 1;
        inv_func(x, c, resid, jac, dx, f);
        if (resid <= -kVERYBIG || jac == 0.0) { xio = x; return 1; }
        x_older = x; x_old = x; dx_old = dx;
      }
    }
    x += damp * dx;
    errx = (c.w0 == 0.) ? fabs(dx_old) : fabs(fdiv(dx_old, fmax(fabs(c.w0), fabs(x))));
    validate_Wp(x_old, x, c);
    dx_old = dx;
    if (errcheck(errx, x, c) && doing_extra == 0 && extracheck(x, c) > 0) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if ((errcheck(errx, x, c) && doing_extra == 0) || (i_extra > extracheck(x, c)) || (n_iter >= (kMAX_NEWT_ITER - 1)))
      keep = false;
    n_iter++;
  }
  if (!isfinite(x) || !isfinite(f) || !isfinite(-2.0 * f)) {
    flag = HARM_UTOPRIMFAILNANRESULT;
    xio = x;
    return 1;
  }
  x = x_old;
  xio = x;
  if (errcheck(errx, x, c)) return 0;
  if (fabs(errx) > kMIN_NEWT_TOL) { flag = HARM_UTOPRIMFAILCONVRET + 4; return 1; }
  return 0;
}

// Setup scalars and the previous-state guess; returns retval contribution of the guess.
// U and prim are alpha-scaled as in Utoprim_jon_nonrelcompat_inputnorestmass.
// compute_setup_quantities: the alpha-scaled invariants D, B^2, (Q.B)^2, Qt^2, Q.n' of U
static __device__ __forceinline__ void inv_invariants(const double* U, const Geo<double>& g, InvC& c, double Qtcon[4],
                                                      double Bcon[4]) {
  c.D = U[HARM_RHO];
  Bcon[0] = 0.;
  Bcon[1] = U[HARM_B1]; Bcon[2] = U[HARM_B2]; Bcon[3] = U[HARM_B3];
  double Bcov[4];
  lower(Bcon, g, Bcov);
  c.Bsq = Bcon[1] * Bcov[1] + Bcon[2] * Bcov[2] + Bcon[3] * Bcov[3];
  double ncov[4] = {-g.alpha, 0., 0., 0.}, ncon[4];
  raise(ncov, g, ncon);
  double Qcovp[4] = {U[HARM_UU], U[HARM_U1], U[HARM_U2], U[HARM_U3]}, Qconp[4];
  raise(Qcovp, g, Qconp);
  Qtcon[0] = 0.0;
#pragma unroll
  for (int j = 1; j < 4; j++) {
    double s = 0.0;
#pragma unroll
    for (int i = 1; i < 4; i++) s += U[HARM_UU + i] * (g.gcon[sym(i, j)] + ncon[i] * ncon[j]);
    Qtcon[j] = s;
  }
  double Qtcov[4];
  lower(Qtcon, g, Qtcov);
  c.Qtsq = Qtcov[0] * Qtcon[0] + Qtcov[1] * Qtcon[1] + Qtcov[2] * Qtcon[2] + Qtcov[3] * Qtcon[3];
  double Qcov[4] = {Qcovp[0] - c.D, Qcovp[1], Qcovp[2], Qcovp[3]}, Qcon[4];
  raise(Qcov, g, Qcon);
  c.QdotB = Qcov[1] * Bcon[1] + Qcov[2] * Bcon[2] + Qcov[3] * Bcon[3];
  c.QdotBsq = c.QdotB * c.QdotB;
  double alpha = g.alpha, alphasq = alpha * alpha;
  double Dfactor = (-g.gcovpert_tt + alphasq * g.betasqoalphasq) / (alphasq + alpha);
  c.Qdotnp = Qconp[0] * ncov[0] + c.D * Dfactor;
}

static __device__ int inv_setup(const double* U, const Geo<double>& g, const double* prim, InvC& c, double Qtcon[4],
                         double Bcon[4], double& Wp_last, int8_t& flag) {
  inv_invariants(U, g, c, Qtcon, Bcon);
  // set_guess_Wp
  double utsq = 0.;
#pragma unroll
  for (int i = 1; i < 4; i++)
#pragma unroll
    for (int j = 1; j < 4; j++) utsq += g.gcov[sym(i, j)] * prim[HARM_U1 + i - 1] * prim[HARM_U1 + j - 1];
  if ((utsq < 0.) && (fabs(utsq) < fabs(-0.9 * c.utsq_too_big))) utsq = 0.0;
  if (!(utsq >= 0. && utsq < c.utsq_too_big)) utsq = 0.0;
  double gammasq = 1. + utsq, gamma = sqrt(gammasq), rho0 = c.D / gamma, u = prim[HARM_UU];
  double p = (c.gam - 1.) * u;
  double bc[4] = {0.0, prim[HARM_B1], prim[HARM_B2], prim[HARM_B3]}, bcv[4];
  lower(bc, g, bcv);
  double bsq = bc[1] * bcv[1] + bc[2] * bcv[2] + bc[3] * bcv[3];
  bsq *= (g.alpha * g.alpha) / gammasq;
  Wp_last = c.D * utsq / (1.0 + gamma) + (u + p) * gammasq;
  double Wpabs = fabs(c.D * utsq) / (1.0 + fabs(gamma)) + (fabs(u) + fabs(p)) * fabs(gammasq) + kSQRTMIN;
  double etaabs = fabs(rho0) + (fabs(u) + fabs(p) + fabs(bsq));
  c.w2 = 1e2 * fabs(rho0);
  if (gammasq * etaabs >= c.w2) {
    double Wpc;
    if (!coldgrhd(c.Qtsq, c.D, Wpc)) { flag = HARM_UTOPRIMFAILCONVUTSQ; Wpc = Wp_last; }
    c.w0 = fmax(fmax(Wpc, Wp_last), Wpabs);
    Wp_last = fmax(2.0 * Wpc, Wp_last);
  } else {
    c.w0 = Wpabs;
  }
  c.w1 = fabs(rho0) + c.w0 + kSQRTMIN;
  return 0;
}

// verify_Wlast and the utsq>=0 guard loop of set_guess_Wp
static __device__ int inv_verify_guess(double& Wp_last, const InvC& c, int8_t& flag) {
  double W_last = Wp_last + c.D;
  if (W_last < -(c.D) || Wp_last < 0) { W_last = -(c.D); Wp_last = 0; }
  for (int inc = 0; vsqgtr1(W_last, c) && inc < 10; inc++) {
    Wp_last *= 10.;
    W_last = Wp_last + c.D;
  }
  for (int attempts = 0;; attempts++) {
    double ut2 = utsq_calc(W_last, c);
    if (ut2 >= 0.0 && ut2 == ut2) break;
    double coldWp = Wp_last;
    coldgrhd(c.Qtsq, c.D, coldWp);
    if (Wp_last < coldWp) Wp_last = coldWp;
    if (attempts > 0) Wp_last = fmax(fmax(fabs(Wp_last) * 10.0, 2.220446049250313e-16 * 100.0 * fabs(c.D)), kKINDASMALL);
    W_last = Wp_last + c.D;
    if (attempts > 1000) { flag = HARM_UTOPRIMFAILCONVGUESSUTSQ; return 1; }
  }
  return 0;
}

// W' -> primitives (Wp2prim), including check_Wp's flags.  prim is alpha-scaled.
static __device__ int inv_finish(double Wp, const InvC& c, const double* Qtcon, const double* Bcon, double* prim, int8_t& flag) {
  if (Wp == kBIG) flag = HARM_UTOPRIMFAILCONVRET + 1;
  else if (Wp <= -(c.D)) flag = HARM_UTOPRIMFAILCONVRET + 1;
  else if (Wp / c.w1 > c.gsq_too_big) flag = HARM_UTOPRIMFAILCONVW;
  double W = Wp + c.D;
  double utsq = utsq_calc(W, c), gammasq = 1.0 + utsq, gamma = sqrt(gammasq);
  double wmrho0 = (Wp - c.D * utsq / (1.0 + gamma)) / gammasq;
  double rho0 = c.D / gamma;
  double p = ((c.gam - 1.0) / c.gam) * wmrho0, u = wmrho0 - p;
  if ((rho0 <= 0.) || ((p < 0.) && !c.cold)) {
    if ((rho0 <= 0.) && (p >= 0.)) flag = HARM_UTOPRIMFAILRHONEG;
    if ((rho0 > 0.) && (p < 0.)) flag = HARM_UTOPRIMFAILUNEG;
    if ((rho0 <= 0.) && (p < 0.)) flag = HARM_UTOPRIMFAILRHOUNEG;
  }
  double out[5];
  out[0] = rho0;
  out[1] = c.cold ? 0.0 : u;
#pragma unroll
  for (int i = 1; i < 4; i++) out[1 + i] = gamma / (W + c.Bsq) * (Qtcon[i] + c.QdotB * Bcon[i] / W);
  bool nan = false;
#pragma unroll
  for (int i = 0; i < 5; i++) nan |= !isfinite(out[i]);
  if (nan) { flag = HARM_UTOPRIMFAILNANRESULT; return 1; }
#pragma unroll
  for (int i = 0; i < 5; i++) prim[i] = out[i];
  return 0;
}

// The inversion split in two: jon_prepare computes everything that does not depend on the
// starting W' (the alpha-scaled setup quantities and the previous-state guess with its
// convergence scales wglobal), jon_solve runs verify_Wlast, the Newton iteration and Wp2prim
// from a given starting W'.  The learned guess runs between the two.
struct JonSetup {
  InvC c;
  double Qtcon[4], Bcon[4];
  double Wp_prev;  // set_guess_Wp's W' from the previous primitive state
  int8_t flag0;    // flag raised by the setup (cold-HD guess without a root)
};

// Utoprim_jon_nonrelcompat_inputnorestmass up to set_guess_Wp, on geometry-free U.
// prim's field components are replaced by U's (as the reference does on entry).
static __device__ __forceinline__ void jon_prepare(bool cold, const double* Ugf, const Geo<double>& g, double* prim,
                                                   double gam, double gammafail, JonSetup& s) {
  double U[NPR], pt[NPR];
  const double alpha = g.alpha;
#pragma unroll
  for (int i = 0; i < NPR; i++) U[i] = alpha * Ugf[i];
#pragma unroll
  for (int i = 0; i < NPR; i++) pt[i] = prim[i];
  pt[HARM_B1] = alpha * Ugf[HARM_B1];
  pt[HARM_B2] = alpha * Ugf[HARM_B2];
  pt[HARM_B3] = alpha * Ugf[HARM_B3];
  prim[HARM_B1] = Ugf[HARM_B1];
  prim[HARM_B2] = Ugf[HARM_B2];
  prim[HARM_B3] = Ugf[HARM_B3];
  s.c.cold = cold;
  s.c.gam = gam;
  s.c.gsq_too_big = gammafail * gammafail;
  s.c.utsq_too_big = (gammafail - 1.0) * (gammafail - 1.0);
  s.flag0 = HARM_UTOPRIMNOFAIL;
  inv_setup(U, g, pt, s.c, s.Qtcon, s.Bcon, s.Wp_prev, s.flag0);
}

// The rest of the inversion from the starting W' `Wp`: prim[RHO..U3] receive the
// primitives on success; flag the outcome; wp_out (optional) the final W'.
// GATED: returns true, with prim and flag untouched, where the first Newton step from Wp
// exceeds `gate` (newton<true>); otherwise the same operations as without GATED.
template <bool GATED = false>
static __device__ __forceinline__ bool jon_solve(const JonSetup& s, double Wp, double* prim, int8_t& flag, int& nstroke,
                                                 double* wp_out = nullptr, double gate = 0.0) {
  int lntries = 0;
  int8_t flag_in = flag;
  flag = s.flag0;
  int retval = inv_verify_guess(Wp, s.c, flag);
  if (GATED && retval == 0) {
    const int r = newton<true>(flag, Wp, s.c, lntries, nstroke, gate);
    if (r == 2) {
      flag = flag_in;
      return true;
    }
    retval += r;
  } else {
    retval += newton(flag, Wp, s.c, lntries, nstroke);
  }
  if (wp_out) *wp_out = Wp;
  double pt[5];
  if (retval == 0) retval = inv_finish(Wp, s.c, s.Qtcon, s.Bcon, pt, flag);
  if (retval == 0) {
#pragma unroll
    for (int i = 0; i <= HARM_U3; i++) prim[i] = pt[i];
  } else {
    if (flag <= 0) flag = (int8_t)(retval + HARM_UTOPRIMFAILCONVRET + 1);
  }
  return false;
}

// Hot or cold Jon inversion on geometry-free U (Utoprim_jon_nonrelcompat_inputnorestmass).
// `wpguess` replaces the previous-state W' when use_guess is set.
static __device__ __forceinline__ void utoprim_jon(bool cold, const double* Ugf, const Geo<double>& g, int8_t& flag, double* prim, double gam,
                            double gammafail, int& nstroke, bool use_guess, double wpguess) {
  JonSetup s;
  jon_prepare(cold, Ugf, g, prim, gam, gammafail, s);
  jon_solve(s, use_guess ? wpguess : s.Wp_prev, prim, flag, nstroke);
}

// Utoprimgen from UEVOLVE U (igdet scales to geometry-free).  Returns the Newton iterations.
static __device__ __forceinline__ int utoprimgen(const double* U, const Geo<double>& g, double igdet, double* pr, int8_t& flag, double gam,
                          double gammafail, bool use_guess, double wpguess, bool* guess_failed) {
  double Ugf[NPR], pr0[NPR];
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) { Ugf[pl] = U[pl] * igdet; pr0[pl] = pr[pl]; }
  int nstroke = 0;
  utoprim_jon(false, Ugf, g, flag, pr, gam, gammafail, nstroke, use_guess, wpguess);
  if (use_guess && flag != HARM_UTOPRIMNOFAIL) {
    // the learned guess did not converge: redo from the previous-state guess
    if (guess_failed) *guess_failed = true;
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) pr[pl] = pr0[pl];
    utoprim_jon(false, Ugf, g, flag, pr, gam, gammafail, nstroke, false, 0.0);
  }
  if (flag) {
    double prhot[NPR], prcold[NPR];
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) { prhot[pl] = pr[pl]; prcold[pl] = pr0[pl]; }
    int8_t cflag = 0;
    utoprim_jon(true, Ugf, g, cflag, prcold, gam, gammafail, nstroke, false, 0.0);
    if (cflag <= 0) {
#pragma unroll
      for (int pl = 0; pl < NPR; pl++) pr[pl] = prcold[pl];
      pr[HARM_UU] = pr0[HARM_UU];
      flag = HARM_UTOPRIMFAILU2AVG1;
    } else {
#pragma unroll
      for (int pl = 0; pl < NPR; pl++) pr[pl] = prhot[pl];
    }
  }
  return nstroke;
}

}  // namespace hb
