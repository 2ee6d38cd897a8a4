/*
 * orc_recon_hi.c -- TEST INFRASTRUCTURE ONLY (CPU oracle; see harm_oracle.h).
 *
 * WENO5 (lim = WENO5BND) centre-to-edge reconstruction of one line, restating
 * eno_line_reconstruct (reconstructeno.c:333) for cvt_type CVT_C2E with the switches of
 * reconstructeno_global.h:
 *   - smoothness indicators of the three 3-point stencils (compute_cf_stencil_weights
 *     reconstructeno.c:1693, order 3), desensitised by sum(u^2)*WENO_EPSILON (USE_NORMU,
 *     desensitise_smoothness_indicators :2001) and normalised to unit sum
 *     (DO_NORMALIZE_SMOOTHNESS_INDICATORS, normalize_array :2292);
 *   - unoptimised weights 1/(beta+WENO_EPSILON)^2 (compute_weights_from_smoothness_indicators
 *     :2211), normalised, passed through limit_weight (:3015, DO_LIMIT_C2E_WEIGHTS) and
 *     normalised again;
 *   - optimal left/right face weights (compute_optimized_cf_stencil_weights :1905,
 *     c2e_optimal_weights_* reconstructeno_staticfuncs_constvars.h:214-226);
 *   - the same for the 2-stencil WENO3 (compute_lower_order_stencil_weights :1300);
 *   - stencil reduction: the ratio of a stencil's weight to its neighbour's weight at
 *     distance 2 gives lower_order_fraction = clamp((min ratio - 1.3)/0.3, 0, 1)
 *     (compute_weights_ratios :2316, DO_OR_STENCIL_REDUCTION=0), and the output mixes
 *     (1-f) WENO5 + f WENO3 (choose_weno_order :2442);
 *   - edge values from the stencil polynomials (eno_cvt :884, c2l/c2r_array2/3 :335-349),
 *     all sums in the symmetric pairwise order of get_sum_of_elements (:2266,
 *     SYMMETRIZE_WENO=1).
 * Not restated: the SMONO monotonicity indicator (DO_SMONO_C2E, interpline.smono.c), which
 * here is taken as 0 everywhere (pure WENO output), the shock / pressure-jump reductions
 * (apply_additional_reduction_to_weights, SHOCKINDICATOR), and the GAMCHECK switch of the
 * ratio thresholds for Lorentz factors above 10.
 *
 * PPM (lim = PARA, WHICHPARA=PARA4): para4 / para4gen (interppoint.para.c:568, :611) with
 * PARA2LIM=MC, JONPARASTEEP=0, JONPARASMOOTH=0, JONPARAREDUCE=0, WHICHLIMITERTOUSEFORLR=0,
 * PARAGENDQALLOWEXTREMUM=0, AVGINPUT=0: MC-limited slopes dq of the cells -1,0,1, face values
 * from paracont (:958, 4th-order average minus ddq/8), then checkparamonotonicity (:1069,
 * NONMONOLIM=0, a6 coefficient 4).
 *
 * Line PPM (lim = PARALINE): pass_1d_line_multipl_paraline (interpline.para.c:8) with the
 * switches of para_and_paraenohybrid.h and definit.h (DOPPMREDUCE=1, DOPPMCONTACTSTEEP=0,
 * JONPARASMOOTH=0, PARALINEUSESMONO=0, NONMONOLIM=0):
 *   - slopes dq[i] = MINMODB(dq2, MINMODB(2 dq1l, 2 dq1r)), the MC limiter with the extremum
 *     allowed (compute_df_line_paraline interpline.c:3463, get_limit_slopes_paraline
 *     interpline.para.c:165 with PARALINE2LIM=MC, PARALINE2EXTREME=1, MINMODGEN
 *     global.nondepnmemonics.h:641);
 *   - continuous face values facecont[i] = (y[i]+y[i-1])/2 - (dq[i]-dq[i-1])/8 (paracont
 *     interppoint.para.c:958, DF2OFMONO);
 *   - cell i: l = facecont[i], r = facecont[i+1], pulled towards y[i] by the flattening
 *     coefficient Fi[i] (paraflatten :1305), then the same checkparamonotonicity as PARA4;
 *   - Fi from the cell's V = sqrt(-g) rho u^dir and total pressure P = p + b^2/2
 *     (get_V_and_P interpline.c:2964, VLINEWITHGDETRHO=1, PLINEWITHFIELD=1) through Ficalc
 *     (interppoint.para.c:1356) and ftilde (:1316), FLASH's flattener with SP0 = 0.75
 *     (get_shock_indicator interpline.c:3114).  The reference's max/min are the functions of
 *     phys.tools.c:2356 (a > b ? a : b and a > b ? b : a), its sign() is copysign(1, a), and
 *     the 1/3 threshold is the long double THIRD (global.nondepnmemonics.h:746).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "harm_oracle.h"
#include "orc_internal.h"

#define WENO_EPS ((500.0 * DBL_EPSILON) * (500.0 * DBL_EPSILON)) /* WENO_EPSILON */

/* get_sum_of_elements, SYMMETRIZE_WENO: pair element i with n-1-i */
static double symsum(int n, const double *a) {
  double s = 0.0;
  int i;
  for (i = 0; i < n / 2; i++) s += a[i] + a[n - 1 - i];
  s += a[i] * (n % 2);
  return s;
}

static double normalize(int n, double eps, double *a) {
  double s = symsum(n, a);
  for (int i = 0; i < n; i++) a[i] /= (s + eps);
  return s;
}

static double limit_weight(int order, double w) {
  double avg = 1.0 / order, w1 = 0.2 * avg, w2 = (1.0 - 0.2) * avg, w3 = (1.0 + 0.2) * avg, w4 = 1.0;
  if (w < w1) return 0.0;
  if (w < w2) return avg * (w - w1) / (w2 - w1);
  if (w < w3) return avg;
  return (w - w3) * (w4 - avg) / (w4 - w3) + avg;
}

/* weights of one cell: w[0..r-1] unoptimised, w[r..2r-1] left face, w[2r..3r-1] right face.
   u points at the cell. */
typedef struct wts {
  double w5[9], w3[6];
  double frac;
} wts;

static void cell_weights(int r, const double *u, double *w) {
  double beta[3];
  if (r == 3) {
    double fd[3], sd[3];
    fd[0] = -(3 * u[0] + u[2]) + 4 * u[1];
    fd[1] = u[1] - u[-1];
    fd[2] = (3 * u[0] + u[-2]) - 4 * u[-1];
    sd[0] = (u[0] + u[2]) - 2 * u[1];
    sd[1] = (u[-1] + u[1]) - 2 * u[0];
    sd[2] = (u[0] + u[-2]) - 2 * u[-1];
    for (int s = 0; s < 3; s++) beta[s] = 13. / 12. * sd[s] * sd[s] + 1. / 4. * fd[s] * fd[s];
  } else {
    double fd[2] = {u[1] - u[0], u[0] - u[-1]};
    for (int s = 0; s < 2; s++) beta[s] = fd[s] * fd[s];
  }
  double u2[5];
  for (int i = -r + 1; i < r; i++) u2[i + r - 1] = u[i] * u[i];
  double normu = symsum(2 * r - 1, u2);
  double eeps = normu * WENO_EPS;
  for (int s = 0; s < r; s++) beta[s] += eeps;
  normalize(r, DBL_MIN, beta);
  for (int s = 0; s < r; s++) {
    double t = beta[s] + WENO_EPS;
    t *= t;
    w[s] = 1. / t;
  }
  normalize(r, 0.0, w);
  for (int s = 0; s < r; s++) w[s] = limit_weight(r, w[s]);
  normalize(r, 0.0, w);
  static const double dl3[3] = {1. / 16., 5. / 8., 5. / 16.}, dr3[3] = {5. / 16., 5. / 8., 1. / 16.};
  static const double dl2[2] = {1. / 4., 3. / 4.}, dr2[2] = {3. / 4., 1. / 4.};
  for (int s = 0; s < r; s++) {
    w[r + s] = w[s] * (r == 3 ? dl3[s] : dl2[s]);
    w[2 * r + s] = w[s] * (r == 3 ? dr3[s] : dr2[s]);
  }
  normalize(r, DBL_MIN, w + r);
  normalize(r, DBL_MIN, w + 2 * r);
}

/* eno_cvt: sum_s w_s * sum_j M[s][j] u[j-s] */
static double cvt(int r, int right, const double *w, const double *u) {
  static const double l3[3][3] = {{15. / 8., -5. / 4., 3. / 8.}, {3. / 8., 3. / 4., -1. / 8.}, {-1. / 8., 3. / 4., 3. / 8.}};
  static const double r3[3][3] = {{3. / 8., 3. / 4., -1. / 8.}, {-1. / 8., 3. / 4., 3. / 8.}, {3. / 8., -5. / 4., 15. / 8.}};
  static const double l2[2][2] = {{3. / 2., -1. / 2.}, {1. / 2., 1. / 2.}};
  static const double r2[2][2] = {{1. / 2., 1. / 2.}, {-1. / 2., 3. / 2.}};
  double upd[3];
  for (int s = 0; s < r; s++) {
    double pts[3];
    for (int j = 0; j < r; j++) {
      double m = (r == 3) ? (right ? r3[s][j] : l3[s][j]) : (right ? r2[s][j] : l2[s][j]);
      pts[j] = m * u[j - s];
    }
    upd[s] = 0.0;
    if (w[s] != 0.0) upd[s] = w[s] * symsum(r, pts);
  }
  return symsum(r, upd);
}

void o_recon_line_weno5(int n, const double *y, double *yl, double *yr) {
  for (int c = 0; c < n; c++) yl[c] = yr[c] = y[c];
  if (n < 9) return;
  wts *W = (wts *)calloc((size_t)n, sizeof(wts));
  for (int c = 2; c < n - 2; c++) {
    cell_weights(3, y + c, W[c].w5);
    cell_weights(2, y + c, W[c].w3);
  }
  for (int c = 4; c < n - 4; c++) {
    /* compute_weights_ratios: LEFT_WEIGHT = 2, RIGHT_WEIGHT = 0, neighbours at c -/+ 2 */
    double rl = (W[c].w5[2] + WENO_EPS) / (W[c - 2].w5[0] + WENO_EPS);
    double rr = (W[c].w5[0] + WENO_EPS) / (W[c + 2].w5[2] + WENO_EPS);
    double ratio = fmin(rl, rr);
    double f = (ratio - 1.3) / (1.6 - 1.3);
    f = fmax(0., fmin(f, 1.0));
    W[c].frac = f;
  }
  for (int c = 4; c < n - 4; c++) {
    double f = W[c].frac;
    double w5[9], w3[6];
    memcpy(w5, W[c].w5, sizeof(w5));
    memcpy(w3, W[c].w3, sizeof(w3));
    int two = (0.0 < f);
    if (two) {
      for (int k = 3; k < 9; k++) w5[k] *= (1. - f);
      for (int k = 0; k < 6; k++) w3[k] *= f;
    }
    double outl = 0.0, outr = 0.0;
    outl += cvt(3, 0, w5 + 3, y + c);
    outr += cvt(3, 1, w5 + 6, y + c);
    if (two) {
      outl += cvt(2, 0, w3 + 2, y + c);
      outr += cvt(2, 1, w3 + 4, y + c);
    }
    yl[c] = (1.0 - 0.0) * outl + 0.0 * y[c];
    yr[c] = (1.0 - 0.0) * outr + 0.0 * y[c];
  }
  free(W);
}

#define MINMODB(a, b) ((fabs(a) < fabs(b)) ? (a) : (b))
#define MINMOD(a, b) (((a) * (b) <= 0) ? 0.0 : MINMODB(a, b))

static void para_monotonicity(const double *y, double *lio, double *rio);

/* para4 of the cell at y[0] (uses y[-2..2]) */
static void para4(const double *y, double *lout, double *rout) {
  double dq1[4], dq2[3], dq[3];
  for (int mm = -1; mm <= 1; mm++) {
    dq1[mm + 1] = (y[mm] - y[mm - 1]);
    dq2[mm + 1] = 0.5 * (y[mm + 1] - y[mm - 1]);
  }
  dq1[3] = (y[2] - y[1]);
  for (int mm = -1; mm <= 1; mm++) {
    double Dqm = 2.0 * dq1[mm + 1], Dqp = 2.0 * dq1[mm + 2], Dqc = dq2[mm + 1];
    dq[mm + 1] = MINMOD(Dqc, MINMOD(Dqm, Dqp));
  }
  double ddql = (dq[1] - dq[0]), ddqr = (dq[2] - dq[1]);
  double l = 0.5 * (y[0] + y[-1]) - ddql * (1.0 / 8.0);
  double r = 0.5 * (y[1] + y[0]) - ddqr * (1.0 / 8.0);
  para_monotonicity(y, &l, &r);
  *lout = l;
  *rout = r;
}

/* checkparamonotonicity (interppoint.para.c:1069) with smooth = 0 and
   PARAGENDQALLOWEXTREMUM = 0 */
static void para_monotonicity(const double *y, double *lio, double *rio) {
  double l = *lio, r = *rio;
  double a6 = 4.0;
  double qa = (r - y[0]) * (y[0] - l), qd = (r - l), qe = a6 * (y[0] - 0.5 * (l + r));
  if (qa <= 0.0) {
    l = y[0];
    r = y[0];
  } else {
    if (qd * (qd - qe) < 0.0) l = (-(2.0 + a6) * r + 2.0 * a6 * y[0]) / (a6 - 2.0);
    else if (qd * (qd + qe) < 0.0) r = (-(2.0 + a6) * l + 2.0 * a6 * y[0]) / (a6 - 2.0);
  }
  *lio = l;
  *rio = r;
}

void o_recon_line_para(int n, const double *y, double *yl, double *yr) {
  for (int c = 0; c < n; c++) yl[c] = yr[c] = y[c];
  for (int c = 2; c < n - 2; c++) para4(y + c, &yl[c], &yr[c]);
}

/* ftilde (interppoint.para.c:1316) of the cell at V[0], P[0]: uses P[-2..2], V[-1], V[1] */
static double paraline_ftilde(const double *V, const double *P) {
  double P2diff = P[2] - P[-2];
  double Pbottom = copysign(1.0, P2diff) / (fabs(P2diff) + O_SMALL);
  double Sp = (P[1] - P[-1]) * Pbottom;
  double m = 10.0 * (Sp - 0.75);          /* SP0 */
  double mn = (1.0 > m) ? m : 1.0;        /* min(1.0, m) */
  double Ft = (0.0 > mn) ? 0.0 : mn;      /* max(0, mn) */
  double a = fabs(P[1]), b = fabs(P[-1]);
  double Ft1 = fabs(P[1] - P[-1]) / (((a > b) ? b : a) + O_SMALL);
  Ft *= (double)((long double)Ft1 >= 0.3333333333333333333333333333333333L);
  double Ft2 = V[1] - V[-1];
  Ft *= (double)(Ft2 <= 0.0);
  return Ft;
}

/* Ficalc (interppoint.para.c:1356): uses V[-3..3], P[-3..3] */
static double paraline_fi(const double *V, const double *P) {
  int signdP = (P[1] - P[-1] > 0) * 2 - 1;
  double f0 = paraline_ftilde(V, P), f1 = paraline_ftilde(V - signdP, P - signdP);
  return (f0 > f1) ? f0 : f1;
}

void o_paraline_flattener(int n, const double *V, const double *P, double *Fi) {
  for (int s = 0; s < n; s++) Fi[s] = 0.0;
  for (int s = 3; s < n - 3; s++) Fi[s] = paraline_fi(V + s, P + s);
}

/* slope of the cell at y[0]: MC with the extremum allowed */
static double paraline_dq(const double *y) {
  double dq1l = y[0] - y[-1], dq1r = y[1] - y[0], dq2 = 0.5 * (y[1] - y[-1]);
  double Dqm = 2.0 * dq1l, Dqp = 2.0 * dq1r, Dqc = dq2;
  return MINMODB(Dqc, MINMODB(Dqm, Dqp));
}

void o_recon_line_paraline(int n, const double *y, const double *Fi, double *yl, double *yr) {
  for (int c = 0; c < n; c++) yl[c] = yr[c] = y[c];
  if (n < 5) return;
  double *dq = (double *)calloc((size_t)n, sizeof(double));
  for (int c = 1; c < n - 1; c++) dq[c] = paraline_dq(y + c);
  for (int c = 2; c < n - 2; c++) {
    double l = 0.5 * (y[c] + y[c - 1]) - (dq[c] - dq[c - 1]) * (1.0 / 8.0);
    double r = 0.5 * (y[c + 1] + y[c]) - (dq[c + 1] - dq[c]) * (1.0 / 8.0);
    double f = Fi ? Fi[c] : 0.0;
    l = f * y[c] + (1.0 - f) * l;
    r = f * y[c] + (1.0 - f) * r;
    para_monotonicity(y + c, &l, &r);
    yl[c] = l;
    yr[c] = r;
  }
  free(dq);
}

void orc_paraline_flattener(int n, const double *V, const double *P, double *Fi) {
  o_paraline_flattener(n, V, P, Fi);
}

void orc_reconstruct_line_paraline(int n, const double *y, const double *V, const double *P, double *pl,
                                   double *pr) {
  double *Fi = (double *)calloc((size_t)n, sizeof(double));
  o_paraline_flattener(n, V, P, Fi);
  o_recon_line_paraline(n, y, Fi, pl, pr);
  free(Fi);
}
