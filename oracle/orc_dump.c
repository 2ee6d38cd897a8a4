/*
 * orc_dump.c -- TEST INFRASTRUCTURE ONLY (CPU oracle; see harm_oracle.h).
 *
 * The 52 columns of one row of the reference's main dump file, dump_content (dump.c:449)
 * with CALCFARADAYANDCURRENTS = 0 and GAMMIEDUMP = 0, for active cell (i, j, k):
 *   ti tj tk, X[1..3] (MKS at CENT), V[1..3] (bl_coord, coord.c:930), the primitives,
 *   pressure, cs2 (cs2_compute_idealgas, idealgaseos.c:48), Sden (compute_entropy_simple,
 *   phys.tools.c:3212, with compute_entropy_idealgas, idealgaseos.c:71), the conserved
 *   variables, divb (SETFDIVBFLUXCTTOTHPRIM, global.fieldmacros.h:383 with :115-244),
 *   ucon, ucov, bcon (bcon_calc phys.tools.c:824), bcov, vmin/vmax of the three directions
 *   (vchar), gdet.
 * P has bounded ghost zones; U (NULL: primtoU of P) in the layout of P.
 */
#include <math.h>
#include <string.h>
#include "harm_oracle.h"
#include "orc_internal.h"

#define O_BIG (1.e+100) /* BIG for doubles (global.depnmemonics.h:492) */

static double o_entropy_simple(double rho0, double u, double gam) {
  if (rho0 < O_SMALL) rho0 = O_SMALL;
  if (u < O_SMALL) u = O_SMALL;
  double pressure = (gam - 1.0) * u, indexn = 1.0 / (gam - 1.0), entropy;
  if (rho0 < O_SMALL && pressure < O_SMALL) entropy = 0.0;
  else if (rho0 < O_SMALL) entropy = 0.0;
  else if (pressure < O_SMALL) entropy = -O_BIG;
  else entropy = rho0 * log(pow(pressure, indexn) / pow(rho0, indexn + 1.0));
  if (!isfinite(entropy)) entropy = -O_BIG * fmax(rho0, O_SMALL);
  return entropy;
}

/* gdet B^pl at extended cell (a, b, e) */
static double o_fg(const orc *o, const double *P, int a, int b, int e, int pl) {
  return P[(size_t)pl * o->cells + oidx(o, a, b, e)] * o->geom[(size_t)HARM_G_GDET * o->plane + (size_t)b * o->g.n1e + a];
}
static double o_afg(const orc *o, const double *P, int a, int b, int e, int pl) { return fabs(o_fg(o, P, a, b, e, pl)); }

typedef double (*o_fgfun)(const orc *, const double *, int, int, int, int);

static double o_avg1(o_fgfun F, const orc *o, const double *P, int a, int b, int e, int pl) {
  return 0.5 * (F(o, P, a, b, e, pl) + F(o, P, a - 1, b, e, pl));
}
static double o_avg2(o_fgfun F, const orc *o, const double *P, int a, int b, int e, int pl) {
  return 0.5 * (F(o, P, a, b, e, pl) + F(o, P, a, b - 1, e, pl));
}
/* AVG_for1/2/3: the averages that live on the corners the divergence differences */
static double o_for1(o_fgfun F, const orc *o, const double *P, int a, int b, int e) {
  int em = (o->g.n3 > 1) ? e - 1 : e;
  return 0.5 * (o_avg2(F, o, P, a, b, e, HARM_B1) + o_avg2(F, o, P, a, b, em, HARM_B1));
}
static double o_for2(o_fgfun F, const orc *o, const double *P, int a, int b, int e) {
  int em = (o->g.n3 > 1) ? e - 1 : e;
  return 0.5 * (o_avg1(F, o, P, a, b, e, HARM_B2) + o_avg1(F, o, P, a, b, em, HARM_B2));
}
static double o_for3(o_fgfun F, const orc *o, const double *P, int a, int b, int e) {
  return 0.5 * (o_avg2(F, o, P, a, b, e, HARM_B3) + o_avg2(F, o, P, a - 1, b, e, HARM_B3));
}

void orc_dump_row(const orc *o, const double *P, const double *U, int i, int j, int k, double *out) {
  const harm_grid *hg = &o->g;
  const int ii = i + hg->ng, jj = j + hg->ng, kk = k + hg->ng3;
  const size_t id = oidx(o, ii, jj, kk);
  ogeom g;
  og_load(o, HARM_LOC_CENT, ii, jj, &g);
  double pr[HARM_NPR];
  for (int p = 0; p < HARM_NPR; p++) pr[p] = P[(size_t)p * o->cells + id];
  int col = 0;
  out[col++] = (double)i;
  out[col++] = (double)j;
  out[col++] = (double)k;
  double X[4], V[4];
  X[0] = 0.0;
  X[1] = hg->startx[1] + (i + 0.5) * hg->dx[1];
  X[2] = hg->startx[2] + (j + 0.5) * hg->dx[2];
  X[3] = hg->startx[3] + (k + 0.5) * hg->dx[3];
  V[1] = hg->R0 + exp(X[1]);
  if (X[2] < 0.5) V[2] = M_PI * X[2] + ((1. - hg->hslope) / 2.) * sin(2. * M_PI * X[2]);
  else V[2] = M_PI - (M_PI * (1.0 - X[2])) + ((1. - hg->hslope) / 2.) * (-sin(2. * M_PI * (1.0 - X[2])));
  V[3] = 2.0 * M_PI * X[3];
  for (int q = 1; q <= 3; q++) out[col++] = X[q];
  for (int q = 1; q <= 3; q++) out[col++] = V[q];
  for (int p = 0; p < HARM_NPR; p++) out[col++] = pr[p];
  const double gam = hg->gam, rho = pr[HARM_RHO], u = pr[HARM_UU];
  const double pressure = (gam - 1.0) * u, h = rho + u + pressure;
  out[col++] = pressure;
  out[col++] = gam * pressure / h;
  out[col++] = o_entropy_simple(rho, u, gam);
  ostate q;
  o_get_state(pr, &g, gam, &q);
  if (U) {
    for (int p = 0; p < HARM_NPR; p++) out[col++] = U[(size_t)p * o->cells + id];
  } else {
    double F[HARM_NPR];
    o_primtoflux(pr, &q, 0, &g, F);
    for (int p = 0; p < HARM_NPR; p++) out[col++] = F[p];
  }
  {
    const int km = (hg->n3 > 1) ? kk - 1 : kk;
    double D1 = o_for1(o_fg, o, P, ii, jj, kk) - o_for1(o_fg, o, P, ii - 1, jj, kk);
    double D2 = o_for2(o_fg, o, P, ii, jj, kk) - o_for2(o_fg, o, P, ii, jj - 1, kk);
    double D3 = o_for3(o_fg, o, P, ii, jj, kk) - o_for3(o_fg, o, P, ii, jj, km);
    double N1 = o_for1(o_afg, o, P, ii, jj, kk) + o_for1(o_afg, o, P, ii - 1, jj, kk);
    double N2 = o_for2(o_afg, o, P, ii, jj, kk) + o_for2(o_afg, o, P, ii, jj - 1, kk);
    double N3 = o_for3(o_afg, o, P, ii, jj, kk) + o_for3(o_afg, o, P, ii, jj, km);
    double norm = 1.0 / (fabs(N1 / hg->dx[1] + N2 / hg->dx[2] + N3 / hg->dx[3]) + O_SMALL);
    out[col++] = fabs((D1 / hg->dx[1] + D2 / hg->dx[2] + D3 / hg->dx[3]) * norm);
  }
  double bcon[4], bcov[4];
  bcon[0] = pr[HARM_B1] * q.ucov[1] + pr[HARM_B2] * q.ucov[2] + pr[HARM_B3] * q.ucov[3];
  for (int m = 1; m <= 3; m++) bcon[m] = (pr[HARM_B1 - 1 + m] + bcon[0] * q.ucon[m]) / q.ucon[0];
  o_lower(bcon, &g, bcov);
  for (int m = 0; m < 4; m++) out[col++] = q.ucon[m];
  for (int m = 0; m < 4; m++) out[col++] = q.ucov[m];
  for (int m = 0; m < 4; m++) out[col++] = bcon[m];
  for (int m = 0; m < 4; m++) out[col++] = bcov[m];
  for (int dir = 1; dir <= 3; dir++) {
    double vmax, vmin;
    o_vchar(pr, &q, dir, &g, gam, &vmax, &vmin);
    out[col++] = vmin;
    out[col++] = vmax;
  }
  out[col++] = g.gdet;
}
