/*
 * host_setup.c -- host-side producers of the inputs of the GRMHD step.
 *
 * This is the part of HARM that runs once before the time loop and is not on the
 * per-timestep path: grid placement (set_points, coord.c:2038), the metric tables
 * (set_grid, set_grid.c:114), the connection (set_connection, set_grid.c:1033) and the
 * Fishbone-Moncrief torus initial state (init_dsandvels_torus,
 * initboundcode/init.fishmon.c:403; field loop :614-732; beta normalisation
 * init.tools.c:745).  The metric is Kerr-Schild in modified Kerr-Schild coordinates
 * (MCOORD KSCOORDS, defcoord LOGRSINTH coord.c:930):
 *     r = R0 + exp(x1),  theta = pi x2 + (1-h)/2 sin(2 pi x2),  phi = 2 pi x3.
 * The inverse metric is written in closed form and the connection uses Ridders'
 * extrapolated central differences of the metric; HARM inverts the metric numerically
 * and differentiates with its DIFFNUMREC scheme.  These tables are inputs of the device
 * path and of the CPU oracle alike.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "harm_b200.h"

#define SINGSMALL 1e-13 /* COORDSINGFIX offset from the poles (init.fishmon.h) */
#define SMALL_D 1e-300  /* SMALL for doubles (global.depnmemonics.h:493) */

static inline int sym_index(int m, int n) {
  static const int t[4][4] = {{0, 1, 2, 3}, {1, 4, 5, 6}, {2, 5, 7, 8}, {3, 6, 8, 9}};
  return t[m][n];
}

int harm_grid_setup(harm_grid *g, int n1, int n2, int n3, int lim, double a,
                    double hslope, double Rout, double cour) {
  /* the radial boundary extrapolates from three cells, the polar one reads the second
     cell from each pole while it rewrites the first */
  if (!g || n1 < 3 || n2 < 4 || n3 < 1) return 1;
  if (lim != HARM_LIM_MC && lim != HARM_LIM_PARA && lim != HARM_LIM_WENO5 && lim != HARM_LIM_PARALINE) return 1;
  memset(g, 0, sizeof(*g));
  g->n1 = n1; g->n2 = n2; g->n3 = n3;
  g->lim = lim;
  /* MAXBND: 4 for MC/PARA/PARALINE, 6 for WENO5BND (initboundcode/init.fishmon.h) */
  g->ng = (lim == HARM_LIM_WENO5) ? 6 : 4;
  g->ng3 = (n3 > 1) ? g->ng : 0;
  g->n1e = n1 + 2 * g->ng;
  g->n2e = n2 + 2 * g->ng;
  g->n3e = n3 + 2 * g->ng3;
  g->a = a;
  g->hslope = hslope;
  g->R0 = 0.0;
  g->Rout = Rout;
  g->Rhor = 1.0 + sqrt(fmax(1.0 - a * a, 0.0)); /* rhor_calc(0), metric.tools.c:1140 */
  /* setihor (coord.c:2334): min(0.1 N1, MAXBND); setRin (coord.c:2346) puts the
     horizon ADJUSTFRACT=0.25 of a cell inside face ihor. */
  int ihor = (n1 * 0.1 > g->ng) ? g->ng : (int)(n1 * 0.1);
  double ftemp = (ihor + 0.25) / (double)n1;
  g->Rin = g->R0 + pow((g->Rhor - g->R0) / pow(Rout - g->R0, ftemp), 1.0 / (1.0 - ftemp));
  g->startx[0] = 0.0;
  g->startx[1] = log(g->Rin - g->R0);
  g->startx[2] = 0.0;
  g->startx[3] = 0.0;
  g->dx[0] = 0.0;
  g->dx[1] = log((Rout - g->R0) / (g->Rin - g->R0)) / n1;
  g->dx[2] = 1.0 / n2;
  g->dx[3] = 1.0 / n3;
  g->gam = 4.0 / 3.0;
  g->cour = cour;
  g->defcon = 1.0;
  g->safe = 1.3;
  g->rho_floor_coef = 1e-6;
  g->u_floor_coef = 1e-8;
  g->gammamax = 25.0;
  g->gammafail = 100.0 * g->gammamax;
  return 0;
}

/* Boyer-Lindquist theta of x2, with both branches of coord.c:953-959 and the
   COORDSINGFIX clamp of coord.c:1443-1452. */
static double theta_of_x2(const harm_grid *g, double x2) {
  double th;
  if (x2 < 0.5)
    th = M_PI * x2 + 0.5 * (1.0 - g->hslope) * sin(2.0 * M_PI * x2);
  else
    th = M_PI - M_PI * (1.0 - x2) - 0.5 * (1.0 - g->hslope) * sin(2.0 * M_PI * (1.0 - x2));
  if (fabs(th) < SINGSMALL) th = (th >= 0) ? SINGSMALL : -SINGSMALL;
  if (fabs(M_PI - th) < SINGSMALL) th = (th >= M_PI) ? M_PI + SINGSMALL : M_PI - SINGSMALL;
  return th;
}

static double dthdx2(const harm_grid *g, double x2) {
  if (x2 < 0.5) return M_PI + (1.0 - g->hslope) * M_PI * cos(2.0 * M_PI * x2);
  return M_PI + (1.0 - g->hslope) * M_PI * cos(2.0 * M_PI * (1.0 - x2));
}

/* covariant MKS metric at (x1,x2) */
static void gcov_mks(const harm_grid *g, double x1, double x2, double gcov[4][4]) {
  double r = g->R0 + exp(x1), th = theta_of_x2(g, x2), a = g->a;
  double cth = cos(th), sth = sin(th), s2 = sth * sth;
  double rho2 = r * r + a * a * cth * cth;
  double z = 2.0 * r / rho2;
  double d[4] = {1.0, r - g->R0, dthdx2(g, x2), 2.0 * M_PI};
  double k[4][4];
  memset(k, 0, sizeof(k));
  k[0][0] = -1.0 + z;
  k[0][1] = k[1][0] = z;
  k[0][3] = k[3][0] = -z * a * s2;
  k[1][1] = 1.0 + z;
  k[1][3] = k[3][1] = -a * s2 * (1.0 + z);
  k[2][2] = rho2;
  k[3][3] = s2 * (rho2 + a * a * s2 * (1.0 + z));
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) gcov[m][n] = k[m][n] * d[m] * d[n];
}

/* one location record: gcov, gcon (closed form), lapse, shift, sqrt(-g) */
static void metric_record(const harm_grid *g, double x1, double x2, double *rec) {
  double r = g->R0 + exp(x1), th = theta_of_x2(g, x2), a = g->a;
  double cth = cos(th), sth = sin(th), s2 = sth * sth;
  double rho2 = r * r + a * a * cth * cth;
  double z = 2.0 * r / rho2;
  double d[4] = {1.0, r - g->R0, dthdx2(g, x2), 2.0 * M_PI};
  double gcov[4][4], kc[4][4];
  gcov_mks(g, x1, x2, gcov);
  memset(kc, 0, sizeof(kc));
  kc[0][0] = -(1.0 + z);
  kc[0][1] = kc[1][0] = z;
  kc[1][1] = (r * r - 2.0 * r + a * a) / rho2;
  kc[1][3] = kc[3][1] = a / rho2;
  kc[2][2] = 1.0 / rho2;
  kc[3][3] = 1.0 / (rho2 * s2);
  for (int m = 0; m < 4; m++)
    for (int n = m; n < 4; n++) {
      rec[HARM_G_GCOV + sym_index(m, n)] = gcov[m][n];
      rec[HARM_G_GCON + sym_index(m, n)] = kc[m][n] / (d[m] * d[n]);
    }
  rec[HARM_G_GCOVPERT_TT] = z;
  double alpha = 1.0 / sqrt(fabs(rec[HARM_G_GCON + 0]));
  rec[HARM_G_ALPHA] = alpha;
  double bsq = 0.0;
  for (int j = 1; j < 4; j++) bsq += rec[HARM_G_GCOV + sym_index(0, j)] * rec[HARM_G_GCON + sym_index(0, j)];
  rec[HARM_G_BETASQOALPHASQ] = bsq;
  for (int j = 1; j < 4; j++) rec[HARM_G_BETA + j - 1] = rec[HARM_G_GCON + sym_index(0, j)] * alpha * alpha;
  double gdet = rho2 * fabs(sth) * d[1] * d[2] * d[3];
  rec[HARM_G_GDET] = gdet;
  rec[HARM_G_IGDET] = ((gdet > 0) - (gdet < 0)) / (fabs(gdet) + SMALL_D);
}

/* Ridders' polynomial extrapolation of central differences of g_{mn} along x1 (dir 1)
   or x2 (dir 2).  Returns all 16 derivative components. */
static void dgcov(const harm_grid *g, double x1, double x2, int dir, double out[4][4]) {
  const int NTAB = 10;
  const double CON = 1.4, CON2 = CON * CON, SAFE = 2.0;
  double h0 = (dir == 1) ? 0.01 * g->dx[1] * 20.0 : 0.01 * g->dx[2] * 20.0;
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) {
      double tab[10][10], err = 1e300, ans = 0.0, hh = h0;
      double gp[4][4], gm[4][4];
      for (int it = 0; it < NTAB; it++) {
        if (dir == 1) { gcov_mks(g, x1 + hh, x2, gp); gcov_mks(g, x1 - hh, x2, gm); }
        else { gcov_mks(g, x1, x2 + hh, gp); gcov_mks(g, x1, x2 - hh, gm); }
        tab[0][it] = (gp[m][n] - gm[m][n]) / (2.0 * hh);
        if (it == 0) { ans = tab[0][0]; hh /= CON; continue; }
        double fac = CON2;
        for (int j = 1; j <= it; j++) {
          tab[j][it] = (tab[j - 1][it] * fac - tab[j - 1][it - 1]) / (fac - 1.0);
          fac *= CON2;
          double errt = fmax(fabs(tab[j][it] - tab[j - 1][it]), fabs(tab[j][it] - tab[j - 1][it - 1]));
          if (errt <= err) { err = errt; ans = tab[j][it]; }
        }
        if (fabs(tab[it][it] - tab[it - 1][it - 1]) >= SAFE * err) break;
        hh /= CON;
      }
      out[m][n] = ans;
    }
}

static void connection_at(const harm_grid *g, double x1, double x2, const double *rec, double *conn) {
  double dg[4][4][4]; /* dg[l][m][n] = d_l g_{mn} */
  memset(dg, 0, sizeof(dg));
  dgcov(g, x1, x2, 1, dg[1]);
  dgcov(g, x1, x2, 2, dg[2]);
  double gcon[4][4];
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) gcon[m][n] = rec[HARM_G_GCON + sym_index(m, n)];
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < 4; l++)
      for (int j = 0; j < 4; j++) {
        double s = 0.0;
        for (int m = 0; m < 4; m++) s += gcon[k][m] * (dg[j][m][l] + dg[l][m][j] - dg[m][l][j]);
        conn[(k * 4 + l) * 4 + j] = 0.5 * s;
      }
}

int harm_geometry_build(const harm_grid *g, double *geom, double *conn, double *aux) {
  if (!g || !geom || !conn || !aux) return 1;
  const int n1e = g->n1e, n2e = g->n2e;
  const size_t plane = (size_t)n1e * n2e;
#pragma omp parallel for schedule(dynamic, 4)
  for (int jj = 0; jj < n2e; jj++) {
    double rec[HARM_NGF], cc[64];
    for (int ii = 0; ii < n1e; ii++) {
      int i = ii - g->ng, j = jj - g->ng;
      double x1c = g->startx[1] + (i + 0.5) * g->dx[1], x1f = g->startx[1] + i * g->dx[1];
      double x2c = g->startx[2] + (j + 0.5) * g->dx[2], x2f = g->startx[2] + j * g->dx[2];
      const double xs[HARM_NLOC][2] = {{x1c, x2c}, {x1f, x2c}, {x1c, x2f}, {x1f, x2f}};
      for (int loc = 0; loc < HARM_NLOC; loc++) {
        metric_record(g, xs[loc][0], xs[loc][1], rec);
        for (int f = 0; f < HARM_NGF; f++) geom[((size_t)loc * HARM_NGF + f) * plane + (size_t)jj * n1e + ii] = rec[f];
        if (loc == HARM_LOC_CENT) {
          connection_at(g, x1c, x2c, rec, cc);
          for (int c = 0; c < 64; c++) conn[(size_t)c * plane + (size_t)jj * n1e + ii] = cc[c];
        }
      }
      double r = g->R0 + exp(x1c);
      aux[(size_t)HARM_AUX_R * plane + (size_t)jj * n1e + ii] = r;
      aux[(size_t)HARM_AUX_RHOFLOOR * plane + (size_t)jj * n1e + ii] = g->rho_floor_coef * pow(r, -1.5);
      aux[(size_t)HARM_AUX_UFLOOR * plane + (size_t)jj * n1e + ii] = g->u_floor_coef * pow(r, -2.5);
    }
  }
  return 0;
}

/* ---------------------------------------------------------------- torus initial state */

/* Keplerian specific angular momentum at the pressure maximum (Fishbone & Moncrief
   1976; lfish_calc, initboundcode/init.fishmon.c:843) */
static double fm_l(double a, double r) {
  double sr = sqrt(r), t1 = a * a - 2.0 * a * sr + r * r;
  double q = sqrt(2.0 * a * sr + (r - 3.0) * r);
  double num = t1 * ((-2.0 * a * r * t1) / q +
                     ((a + (r - 2.0) * sr) * (r * r * r + a * a * (2.0 + r))) /
                         sqrt(1.0 + 2.0 * a / pow(r, 1.5) - 3.0 / r));
  return num / (r * r * r * q * (a * a + (r - 2.0) * r));
}

/* ln(h) of the FM torus relative to its inner edge rin (equatorial) */
static double fm_lnh(double a, double l, double r, double th, double rin) {
  double sth = sin(th), cth = cos(th);
  double DD = r * r - 2.0 * r + a * a;
  double AA = (r * r + a * a) * (r * r + a * a) - DD * a * a * sth * sth;
  double SS = r * r + a * a * cth * cth;
  double DDin = rin * rin - 2.0 * rin + a * a;
  double AAin = (rin * rin + a * a) * (rin * rin + a * a) - DDin * a * a;
  double SSin = rin * rin;
  double f = 1.0 + 4.0 * l * l * SS * SS * DD / (AA * AA * sth * sth);
  double fin = 1.0 + 4.0 * l * l * SSin * SSin * DDin / (AAin * AAin);
  return 0.5 * log((1.0 + sqrt(f)) / (SS * DD / AA)) - 0.5 * sqrt(f) - 2.0 * a * r * l / AA -
         (0.5 * log((1.0 + sqrt(fin)) / (SSin * DDin / AAin)) - 0.5 * sqrt(fin) - 2.0 * a * rin * l / AAin);
}

/* splitmix64: the seeded generator of the perturbation */
static double rng_uniform(uint64_t *s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (z >> 11) * (1.0 / 9007199254740992.0);
}

/* b^2 of a primitive vector with a CENT record (bsq_calc_fromq_rel4vel,
   phys.tools.c:1392) */
static double host_bsq(const double *pr, const double *rec) {
  double gcov[4][4];
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) gcov[m][n] = rec[HARM_G_GCOV + sym_index(m, n)];
  double qsq = 0.0;
  for (int m = 1; m < 4; m++)
    for (int n = 1; n < 4; n++) qsq += gcov[m][n] * pr[HARM_U1 + m - 1] * pr[HARM_U1 + n - 1];
  double gamma = sqrt(1.0 + fmax(qsq, 0.0));
  double ucon[4], ucov[4];
  ucon[0] = gamma / rec[HARM_G_ALPHA];
  for (int j = 1; j < 4; j++) ucon[j] = pr[HARM_U1 + j - 1] - ucon[0] * rec[HARM_G_BETA + j - 1];
  for (int m = 0; m < 4; m++) {
    ucov[m] = 0;
    for (int n = 0; n < 4; n++) ucov[m] += gcov[m][n] * ucon[n];
  }
  double Bsq = 0.0, udotB = 0.0;
  for (int m = 1; m < 4; m++) {
    double Bcov = 0;
    for (int n = 1; n < 4; n++) Bcov += gcov[m][n] * pr[HARM_B1 + n - 1];
    Bsq += pr[HARM_B1 + m - 1] * Bcov;
    udotB += pr[HARM_B1 + m - 1] * ucov[m];
  }
  return (Bsq + udotB * udotB) / (ucon[0] * ucon[0]);
}

int harm_torus_init(const harm_grid *g, const double *geom, const double *aux,
                    double beta_min, uint64_t seed, double *P) {
  if (!g || !geom || !aux || !P) return 1;
  const double a = g->a, gam = g->gam, kappa = 1e-3, rin = 6.0, rmax = 12.0;
  const double l = fm_l(a, rmax);
  const int n1e = g->n1e, n2e = g->n2e, n3e = g->n3e;
  const size_t plane = (size_t)n1e * n2e, cells = plane * n3e;
  double *rho2d = (double *)calloc(plane, sizeof(double));
  double *u2d = (double *)calloc(plane, sizeof(double));
  double *up2d = (double *)calloc(plane, sizeof(double)); /* BL u^phi, 0 outside */
  int *in2d = (int *)calloc(plane, sizeof(int));
  double *A = (double *)calloc(plane, sizeof(double));
  if (!rho2d || !u2d || !up2d || !in2d || !A) return 2;
  double rhomax = 0.0;
  for (int jj = 0; jj < n2e; jj++)
    for (int ii = 0; ii < n1e; ii++) {
      int i = ii - g->ng, j = jj - g->ng;
      double x1 = g->startx[1] + (i + 0.5) * g->dx[1], x2 = g->startx[2] + (j + 0.5) * g->dx[2];
      double r = g->R0 + exp(x1), th = theta_of_x2(g, x2);
      size_t c = (size_t)jj * n1e + ii;
      double lnh = (r >= rin) ? fm_lnh(a, l, r, th, rin) : 1.0;
      if (lnh < 0.0 || r < rin) continue;
      double hm1 = exp(lnh) - 1.0;
      double rho = pow(hm1 * (gam - 1.0) / (kappa * gam), 1.0 / (gam - 1.0));
      double sth = sin(th), cth = cos(th);
      double DD = r * r - 2.0 * r + a * a;
      double AA = (r * r + a * a) * (r * r + a * a) - DD * a * a * sth * sth;
      double SS = r * r + a * a * cth * cth;
      double expm2chi = SS * SS * DD / (AA * AA * sth * sth);
      double up1 = sqrt((-1.0 + sqrt(1.0 + 4.0 * l * l * expm2chi)) / 2.0);
      double up = 2.0 * a * r * sqrt(1.0 + up1 * up1) / sqrt(AA * SS * DD) + sqrt(SS / AA) * up1 / sth;
      rho2d[c] = rho;
      u2d[c] = kappa * pow(rho, gam) / (gam - 1.0);
      up2d[c] = up;
      in2d[c] = 1;
      if (i >= 0 && i < g->n1 && j >= 0 && j < g->n2 && rho > rhomax) rhomax = rho;
    }
  if (rhomax <= 0.0) { free(rho2d); free(u2d); free(up2d); free(in2d); free(A); return 3; }
  /* normalise rho_max = 1 (normalize_densities) */
  double umax = 0.0;
  for (size_t c = 0; c < plane; c++) {
    rho2d[c] /= rhomax;
    u2d[c] /= rhomax;
  }
  /* vector potential at CORN3 from the cell-averaged density, q = rho_av/rho_max - 0.2 */
  for (int jj = 1; jj < n2e; jj++)
    for (int ii = 1; ii < n1e; ii++) {
      double rav = 0.25 * (rho2d[(size_t)jj * n1e + ii] + rho2d[(size_t)(jj - 1) * n1e + ii] +
                           rho2d[(size_t)jj * n1e + ii - 1] + rho2d[(size_t)(jj - 1) * n1e + ii - 1]);
      double q = rav - 0.2;
      A[(size_t)jj * n1e + ii] = q > 0.0 ? q : 0.0;
    }
  /* cell states, all k (the torus is axisymmetric; the perturbation is not) */
  uint64_t st = seed;
  double bsqmax = 0.0, pgmax = 0.0;
  for (int kk = 0; kk < n3e; kk++)
    for (int jj = 0; jj < n2e; jj++)
      for (int ii = 0; ii < n1e; ii++) {
        size_t c = (size_t)jj * n1e + ii, idx = (size_t)kk * plane + c;
        double rec[HARM_NGF];
        for (int f = 0; f < HARM_NGF; f++) rec[f] = geom[((size_t)HARM_LOC_CENT * HARM_NGF + f) * plane + c];
        double r = aux[HARM_AUX_R * plane + c];
        double pr[HARM_NPR] = {0};
        int i = ii - g->ng, j = jj - g->ng, k = kk - g->ng3;
        int active = (i >= 0 && i < g->n1 && j >= 0 && j < g->n2 && k >= 0 && k < g->n3);
        if (in2d[c]) {
          /* BL u^t from normalisation with u^r=u^theta=0; for u^r=0 the Kerr-Schild
             components equal the Boyer-Lindquist ones */
          double x2 = g->startx[2] + (j + 0.5) * g->dx[2];
          double th = theta_of_x2(g, x2), sth = sin(th), cth = cos(th);
          double SS = r * r + a * a * cth * cth, DD = r * r - 2.0 * r + a * a;
          double AA = (r * r + a * a) * (r * r + a * a) - DD * a * a * sth * sth;
          double gtt = -(1.0 - 2.0 * r / SS), gtp = -2.0 * a * r * sth * sth / SS, gpp = AA * sth * sth / SS;
          double up = up2d[c];
          double qa = gtt, qb = 2.0 * gtp * up, qc = gpp * up * up + 1.0;
          double ut = (-qb - sqrt(qb * qb - 4.0 * qa * qc)) / (2.0 * qa);
          double uconp[4] = {ut, 0.0, 0.0, up / (2.0 * M_PI)};
          pr[HARM_RHO] = rho2d[c];
          pr[HARM_UU] = u2d[c];
          if (active) pr[HARM_UU] *= 1.0 + 0.04 * (rng_uniform(&st) - 0.5);
          for (int jv = 1; jv < 4; jv++) pr[HARM_U1 + jv - 1] = uconp[jv] + uconp[0] * rec[HARM_G_BETA + jv - 1];
        } else {
          pr[HARM_RHO] = 1e-4 * pow(r, -1.5);
          pr[HARM_UU] = 1e-6 * pow(r, -2.5);
        }
        if (ii + 1 < n1e && jj + 1 < n2e) {
          double gd = rec[HARM_G_GDET];
          double A00 = A[c], A10 = A[c + 1], A01 = A[c + n1e], A11 = A[c + n1e + 1];
          pr[HARM_B1] = -(A00 - A01 + A10 - A11) / (2.0 * g->dx[2] * gd);
          pr[HARM_B2] = (A00 + A01 - A10 - A11) / (2.0 * g->dx[1] * gd);
        }
        for (int pl = 0; pl < HARM_NPR; pl++) P[(size_t)pl * cells + idx] = pr[pl];
        if (active) {
          double pg = (gam - 1.0) * pr[HARM_UU];
          if (pg > pgmax) pgmax = pg;
          double bsq = host_bsq(pr, rec);
          if (bsq > bsqmax) bsqmax = bsq;
          if (pr[HARM_UU] > umax) umax = pr[HARM_UU];
        }
      }
  /* beta normalisation: beta_act = p_gas,max / (b^2_max/2), B *= sqrt(beta_act/beta_min) */
  if (bsqmax > 0.0) {
    double norm = sqrt((pgmax / (0.5 * bsqmax)) / beta_min);
    for (int pl = HARM_B1; pl <= HARM_B3; pl++)
      for (size_t c = 0; c < cells; c++) P[(size_t)pl * cells + c] *= norm;
  }
  /* floors at t=0 */
  for (int kk = 0; kk < n3e; kk++)
    for (size_t c = 0; c < plane; c++) {
      size_t idx = (size_t)kk * plane + c;
      double rf = aux[HARM_AUX_RHOFLOOR * plane + c], uf = aux[HARM_AUX_UFLOOR * plane + c];
      if (P[(size_t)HARM_RHO * cells + idx] < rf) P[(size_t)HARM_RHO * cells + idx] = rf;
      if (P[(size_t)HARM_UU * cells + idx] < uf) P[(size_t)HARM_UU * cells + idx] = uf;
    }
  free(rho2d); free(u2d); free(up2d); free(in2d); free(A);
  return 0;
}
