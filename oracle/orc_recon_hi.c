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
 *     (compute_weights_ratios :2311, DO_OR_STENCIL_REDUCTION=0), raised where the cell's
 *     momentum-flux jump dP exceeds 0.25 to its neighbours' fractions
 *     (apply_additional_reduction_to_weights :795, DO_REDUCE_POST_SHOCK/PRE_SHOCK,
 *     REDUCE_DP_FRACTION 0.5; dP from compute_df_line_new interpline.c:3557), and the output
 *     mixes (1-f) WENO5 + f WENO3 (choose_weno_order :2442);
 *   - the SMONO monotonicity indicator m of the 5-point polynomial (DO_SMONO_C2E,
 *     compute_mono_indicator_point_eno5 interpline.smono.c:517): m = 1 gives the 5-point
 *     edge values, m in (0,1) blends the cell's WENO5 weights towards equal weights
 *     (mono_adjust_unoptimized_weights :852) and the output towards the 5-point values;
 *   - edge values from the stencil polynomials (eno_cvt :884, c2l/c2r_array2/3 :335-349),
 *     all sums in the symmetric pairwise order of get_sum_of_elements (:2266,
 *     SYMMETRIZE_WENO=1).
 * GAMCHECK (the a2c ratio thresholds for large Lorentz factors, reconstructeno.c:303) is 0 in
 * this build (VSQ is not interpolated).
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
   u points at the cell; m is the cell's SMONO indicator. */
typedef struct wts {
  double w5[9], w3[6];
  double frac, m;
} wts;

static void cell_weights(int r, double m, const double *u, double *w) {
  double beta[3];
  /* compute_cf_stencil_weights (reconstructeno.c:1693): a monotone cell (indicator 1) takes
     equal weights, and its face weights are never formed (its edges are the 5-point values) */
  if (m == 1) {
    for (int s = 0; s < r; s++) w[s] = 1.0 / r;
    return;
  }
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
  /* mono_adjust_unoptimized_weights (:446): a partly monotone cell moves its WENO5 weights
     towards equal ones */
  if (r == 3 && m > 0.0 && m < 1.0)
    for (int s = 0; s < r; s++) w[s] = (1.0 - m) * w[s] + m * (1.0 / r);
}

/* face weights: the unoptimised weights times the optimal ones, normalised
   (compute_optimized_cf_stencil_weights :1905) */
static void face_weights(int r, double *w) {
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

/* SMONO indicator of the 5-point polynomial through u[-2..2] (compute_mono_indicator_point_eno5
   interpline.smono.c:517, SMONO_EPSILON = 500 DBL_EPSILON): 1 where the edge derivatives of
   orders 1..3 agree in sign on both sides and are well above round-off, 0 at an extremum or
   inflection, linear in between (SMONO_DO_SMOOTH_TRANSITION) */
static double smono_indicator(const double *y) {
  double ld[4], rd[4], md[4], minabs = 1.e+100;
  ld[1] = (((-3 * y[-2] + y[2]) + (-10 * y[-1] - 6 * y[1])) + 18 * y[0]) / 12.;
  ld[2] = (((11 * y[-2] - y[2]) + (-20 * y[-1] + 4 * y[1])) + 6 * y[0]) / 12.;
  ld[3] = (((-3 * y[-2] - y[2]) + (10 * y[-1] + 6 * y[1])) - 12 * y[0]) / 2.;
  rd[1] = (((-y[-2] + 3 * y[2]) + (6 * y[-1] + 10 * y[1])) - 18 * y[0]) / 12.;
  rd[2] = (((-y[-2] + 11 * y[2]) + (4 * y[-1] - 20 * y[1])) + 6 * y[0]) / 12.;
  rd[3] = (((y[-2] + 3 * y[2]) - (6 * y[-1] + 10 * y[1])) + 12 * y[0]) / 2.;
#define SMINMODB(a, b) ((fabs(a) < fabs(b)) ? (a) : (b))
#define SMINMOD(a, b) (((a) * (b) <= 0) ? 0.0 : SMINMODB(a, b))
  ld[1] = SMINMOD(ld[1], y[-1] - y[-2]);
  rd[1] = SMINMOD(rd[1], y[2] - y[1]);
  for (int n = 1; n <= 3; n++) {
    md[n] = SMINMOD(ld[n], rd[n]);
    minabs = (minabs < fabs(md[n])) ? minabs : fabs(md[n]);
  }
  double norm = fabs(y[0]) + ((fabs(y[-1]) + fabs(y[1])) + (fabs(y[-2]) + fabs(y[2])));
  double cutoff = norm * (500.0 * DBL_EPSILON) + DBL_MIN;
  double v = (minabs - 0.0) / (cutoff - 0.0);
  v = (1. < v) ? 1. : v;
  return (0. > v) ? 0. : v;
}

/* the 5-point interpolation of the left or right edge (c2e_simple_eno reconstructeno.c:984,
   c2l_array5 / c2r_array5 row 2 reconstructeno_staticfuncs_constvars.h:321-333) */
static double edge5(int right, const double *y) {
  static const double cl[5] = {-5. / 128., 15. / 32., 45. / 64., -5. / 32., 3. / 128.};
  static const double cr[5] = {3. / 128., -5. / 32., 45. / 64., 15. / 32., -5. / 128.};
  double d[5];
  for (int i = -2; i <= 2; i++) d[i + 2] = (right ? cr : cl)[i + 2] * y[i];
  return symsum(5, d);
}

/* the momentum-flux jump indicator of each cell of a line (compute_df_line_new
   interpline.c:3557, from the cell-centre state get_stateforinterpline phys.c:76):
   par = |(1 + u_t) u^dir|, veff = sign(sqrt(-g) rho u^dir) par / (sqrt(par) + SMALL),
   upar = |(u + p + b^2)(|u^dir| u_t) + p + b^2/2 - b^dir b_t|, and
   dP = (|rho (veff[+1] - veff[-1])^2| + |upar[+1] - upar[-1]|) / (|rho par| + |upar| + SMALL)
   for the cells 1..n-2 (0 at the two ends, which no reconstruction reads) */
void o_weno_dp_line(int n, int dir, const double *pr, const ogeom *g, double gam, double *dP) {
  const double SMALL = 1.e-300;
  double *par = (double *)malloc(sizeof(double) * 3 * (size_t)n), *veff = par + n, *upar = par + 2 * n;
  for (int s = 0; s < n; s++) {
    double p[HARM_NPR];
    for (int q = 0; q < HARM_NPR; q++) p[q] = pr[(size_t)q * n + s];
    ostate q;
    o_get_state(p, &g[s], gam, &q);
    double bcon[4], bcov[4];
    bcon[0] = p[HARM_B1] * q.ucov[1] + p[HARM_B2] * q.ucov[2] + p[HARM_B3] * q.ucov[3];
    for (int j = 1; j <= 3; j++) bcon[j] = (p[HARM_B1 - 1 + j] + bcon[0] * q.ucon[j]) / q.ucon[0];
    o_lower(bcon, &g[s], bcov);
    double pgas = q.pressure;
    double V = g[s].gdet * p[HARM_RHO] * q.ucon[dir];
    double btt = -bcon[dir] * bcov[0];
    double ptot = pgas + 0.5 * q.bsq;
    par[s] = fabs(q.plus1ud0 * q.ucon[dir]);
    veff[s] = copysign(1.0, V) * par[s] / (sqrt(par[s]) + SMALL);
    upar[s] = fabs((p[HARM_UU] + pgas + q.bsq) * (fabs(q.ucon[dir]) * q.ucov[0]) + ptot + btt);
  }
  dP[0] = dP[n - 1] = 0.0;
  for (int s = 1; s < n - 1; s++) {
    double rho = pr[(size_t)HARM_RHO * n + s], dv = veff[s + 1] - veff[s - 1];
    dP[s] = (fabs(rho * dv * dv) + fabs(upar[s + 1] - upar[s - 1])) / (fabs(rho * par[s]) + fabs(upar[s]) + SMALL);
  }
  free(par);
}

void o_recon_line_weno5(int n, const double *y, const double *dP, double *yl, double *yr) {
  for (int c = 0; c < n; c++) yl[c] = yr[c] = y[c];
  if (n < 9) return;
  wts *W = (wts *)calloc((size_t)n, sizeof(wts));
  for (int c = 2; c < n - 2; c++) {
    W[c].m = smono_indicator(y + c);
    cell_weights(3, W[c].m, y + c, W[c].w5);
    cell_weights(2, W[c].m, y + c, W[c].w3);
  }
  for (int c = 4; c < n - 4; c++) {
    /* compute_weights_ratios: LEFT_WEIGHT = 2, RIGHT_WEIGHT = 0, neighbours at c -/+ 2; the
       ratio is formed in long double, as WENO_EPSILON is a long double constant there */
    const long double eps = (500.0L * DBL_EPSILON) * (500.0L * DBL_EPSILON);
    double rl = (double)((W[c].w5[2] + eps) / (W[c - 2].w5[0] + eps));
    double rr = (double)((W[c].w5[0] + eps) / (W[c + 2].w5[2] + eps));
    double ratio = fmin(rl, rr);
    double f = (ratio - 1.3) / (1.6 - 1.3);
    f = fmax(0., fmin(f, 1.0));
    W[c].frac = f;
  }
  /* apply_additional_reduction_to_weights (reconstructeno.c:795; DO_REDUCE_POST_SHOCK and
     DO_REDUCE_PRE_SHOCK, REDUCE_DP_FRACTION = 0.5): where the cell's |dP| exceeds 0.25 the
     reduction of either neighbour, scaled by min((|dP| - 0.25)/0.25, 1), is taken if larger;
     the neighbours' fractions are the ones before this step */
  double *lof = (double *)malloc(sizeof(double) * (size_t)n);
  for (int c = 0; c < n; c++) lof[c] = W[c].frac;
  if (dP) {
    for (int c = 5; c < n - 5; c++) {
      double ss = (fabs(dP[c]) - 0.5 * 0.5) / (0.5 * 0.5);
      ss = (ss < 1.) ? ss : 1.;
      double l = W[c].frac, t = ss * W[c + 1].frac;
      l = (l > t) ? l : t;
      t = ss * W[c - 1].frac;
      lof[c] = (l > t) ? l : t;
    }
  }
  for (int c = 4; c < n - 4; c++) {
    const double m = W[c].m;
    double y5l = 0.0, y5r = 0.0;
    if (m != 0) {
      y5l = edge5(0, y + c);
      y5r = edge5(1, y + c);
    }
    if (m >= 1.0) {  /* the monotone cell's edges are the 5-point values */
      yl[c] = y5l;
      yr[c] = y5r;
      continue;
    }
    double f = lof[c];
    double w5[9], w3[6];
    memcpy(w5, W[c].w5, sizeof(w5));
    memcpy(w3, W[c].w3, sizeof(w3));
    face_weights(3, w5);
    face_weights(2, w3);
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
    yl[c] = (1.0 - m) * outl + m * y5l;
    yr[c] = (1.0 - m) * outr + m * y5r;
  }
  free(lof);
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
