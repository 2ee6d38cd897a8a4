/*
 * orc_bound.c -- TEST INFRASTRUCTURE ONLY (CPU oracle; see harm_oracle.h).
 *
 * bound_prim() of the torus problem (step_ch.c:1332 -> bound_anyprim -> bound_prim_user_dir,
 * initboundcode/bounds.fishmon.c:15, per direction 1, 2, 3), restated from bounds.tools.c for
 * the build's configuration (all primitives at CENT, NPRBOUND = 8, one CPU):
 *   x1 inner FREEOUTFLOW and x1 outer OUTFLOW: extrapfunc (bounds.tools.c:1417, the
 *     HORIZONEXTRAP = OUTEREXTRAP = 3 branch, :15-18) from the three cells next to the
 *     boundary; at the outer boundary then inflow_check_rel4vel and limit_gamma (:337);
 *   x2 POLARAXIS at both poles: reflection with U2, B2 negated in the same phi plane
 *     (bound_x2dn_polaraxis :751; the transfer across the pole of
 *     bound_x2dn_polaraxis_full3d needs special3dspc, initbase.c:1501, which a build without
 *     MPI leaves off since periodicx3 = 0, init.tools.c:46-50), then poledeath (:2004) on the
 *     ghost cell and the first
 *     active cell next to the pole (POLEDEATH 1, POLEINTERPTYPE 3, DEATHEXPANDAMOUNT 0,
 *     AVERAGEINRADIUS 0) and POLEGAMMADEATH's Lorentz-factor limit there;
 *   x3 PERIODIC (bound_x3_periodic :1114).
 * Loop ranges of set_boundloop (initbase.boundloop.c:130): the x1 boundary over active j, k;
 * the x2 boundary over all i (ghosts included) and active k; the x3 boundary over all i, j.
 * `nb` is the number of ghost layers filled: all of them (BOUNDPRIMTYPE) or one
 * (BOUNDPRIMSIMPLETYPE, set_numbnd initbase.boundloop.c:65).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "harm_oracle.h"
#include "orc_internal.h"

#define MINMODB(a, b) ((fabs(a) < fabs(b)) ? (a) : (b))
#define MINMOD(a, b) (((a) * (b) <= 0) ? 0.0 : MINMODB(a, b))

static inline double *cellp(const orc *o, double *P, int pl, int i, int j, int k) {
  return P + (size_t)pl * o->cells + oidx(o, i + o->g.ng, j + o->g.ng, k + o->g.ng3);
}

static inline void cent(const orc *o, int i, int j, ogeom *g) {
  og_load(o, HARM_LOC_CENT, i + o->g.ng, j + o->g.ng, g);
}

/* x2 coordinate of cell j's centre and of face j (coord() coord.c:2491) */
static inline double x2c(const harm_grid *g, int j) { return g->startx[2] + (j + 0 + 0.5) * g->dx[2]; }
static inline double x2f(const harm_grid *g, int j) { return g->startx[2] + (j + 0) * g->dx[2]; }

/* extrapfunc (bounds.tools.c:1417) for the line (j,k): the ghost cells i of [ilo, ihi] from
   the reference cells ri, ri2, ri3 (signdq +1 at the inner, -1 at the outer boundary) */
static void extrap_line(const orc *o, double *P, int j, int k, int ri, int ri2, int ri3, double signdq,
                        int ilo, int ihi) {
  ogeom gr, g2, g3;
  cent(o, ri, j, &gr);
  cent(o, ri2, j, &g2);
  cent(o, ri3, j, &g3);
  double p1[HARM_NPR], p2[HARM_NPR], p3[HARM_NPR];
  for (int pl = 0; pl < HARM_NPR; pl++) {
    p1[pl] = *cellp(o, P, pl, ri, j, k);
    p2[pl] = *cellp(o, P, pl, ri2, j, k);
    p3[pl] = *cellp(o, P, pl, ri3, j, k);
  }
  double Bd3 = 0.0, Bd3ri2 = 0.0, Bd3ri3 = 0.0;
  for (int jj = 1; jj <= 3; jj++) Bd3 += p1[HARM_B1 + jj - 1] * gr.gcov[3][jj];
  for (int jj = 1; jj <= 3; jj++) Bd3ri2 += p2[HARM_B1 + jj - 1] * g2.gcov[3][jj];
  for (int jj = 1; jj <= 3; jj++) Bd3ri3 += p3[HARM_B1 + jj - 1] * g3.gcov[3][jj];
  double Dqp = Bd3ri3 - Bd3ri2, Dqm = Bd3ri2 - Bd3, Dqc = Bd3ri3 - Bd3;
  const double dqBd3 = signdq * MINMOD(MINMOD(Dqp, Dqm), Dqc);
  double ucref[4], ucref2[4], gam, qsq;
  o_ucon(p1, &gr, ucref, &gam, &qsq);
  o_ucon(p2, &g2, ucref2, &gam, &qsq);
  double dq[HARM_NPR], dqlog[HARM_NPR], dqgd[HARM_NPR];
  for (int pl = 0; pl < HARM_NPR; pl++) {
    Dqp = p3[pl] - p2[pl];
    Dqm = p2[pl] - p1[pl];
    Dqc = p3[pl] - p1[pl];
    dq[pl] = signdq * MINMOD(MINMOD(Dqp, Dqm), Dqc);
  }
  for (int pl = 0; pl < HARM_NPR; pl++) {
    Dqp = log(O_SMALL + fabs(p3[pl])) - log(O_SMALL + fabs(p2[pl]));
    Dqm = log(O_SMALL + fabs(p2[pl])) - log(O_SMALL + fabs(p1[pl]));
    Dqc = log(O_SMALL + fabs(p3[pl])) - log(O_SMALL + fabs(p1[pl]));
    dqlog[pl] = signdq * MINMOD(MINMOD(Dqp, Dqm), Dqc);
  }
  for (int pl = 0; pl < HARM_NPR; pl++) {
    Dqp = g3.gdet * p3[pl] - g2.gdet * p2[pl];
    Dqm = g2.gdet * p2[pl] - gr.gdet * p1[pl];
    Dqc = g3.gdet * p3[pl] - gr.gdet * p1[pl];
    dqgd[pl] = signdq * MINMOD(MINMOD(Dqp, Dqm), Dqc);
  }
  /* the slopes of u and the velocities fade out where u^t jumps between ri and ri2
     (XDQFRAC1 0.1 .. XDQFRAC2 0.2) */
  const double xdqfrac = fabs(ucref[0] - ucref2[0]) / ucref[0];
  double ydqfrac;
  if (xdqfrac < 0.1) ydqfrac = 0.0;
  else if (xdqfrac < 0.2) ydqfrac = (0.0 + (1.0 - 0.0) / (0.2 - 0.1) * (xdqfrac - 0.1));
  else ydqfrac = 1.0;
  for (int jj = 0; jj < 4; jj++) {
    dq[HARM_UU + jj] = dq[HARM_UU + jj] * (1.0 - ydqfrac);
    dqlog[HARM_UU + jj] = dqlog[HARM_UU + jj] * (1.0 - ydqfrac);
    dqgd[HARM_UU + jj] = dqgd[HARM_UU + jj] * (1.0 - ydqfrac);
  }
  const double powerratio = (1.0 + (0.1));
  for (int i = ilo; i <= ihi; i++) {
    ogeom gi;
    cent(o, i, j, &gi);
    const double di = (double)(i - ri);
    double p[HARM_NPR];
    for (int pl = 0; pl < HARM_NPR; pl++) p[pl] = p1[pl];
    for (int pl = HARM_RHO; pl <= HARM_UU; pl++) {
      double ftemp = exp(-signdq * dqlog[pl]) - powerratio, mydqlog;
      if (ftemp >= 0.0) mydqlog = log(powerratio) / (-signdq);
      else mydqlog = dqlog[pl];
      p[pl] = exp(log(O_SMALL + fabs(p1[pl])) + mydqlog * di);
    }
    for (int pl = HARM_U1; pl <= HARM_U3; pl++) p[pl] = p1[pl] + dq[pl] * di;
    for (int pl = HARM_B1; pl <= HARM_B2; pl++) {
      double igd = copysign(1.0, gi.gdet) / (fabs(gi.gdet) + O_SMALL);
      p[pl] = (p1[pl] * fabs(gr.gdet + dqgd[pl] * di)) * igd;
    }
    {
      const double Bu1 = p[HARM_B1], Bu2 = p[HARM_B2];
      const double gcon03 = gi.gcon[0][3], gcon13 = gi.gcon[1][3], gcon23 = gi.gcon[2][3], gcon33 = gi.gcon[3][3];
      const double gcov01 = gi.gcov[0][1], gcov02 = gi.gcov[0][2], gcov11 = gi.gcov[1][1], gcov12 = gi.gcov[1][2];
      const double gcov21 = gcov12, gcov22 = gi.gcov[2][2], gcov03 = gi.gcov[0][3], gcov13 = gi.gcov[1][3],
                   gcov23 = gi.gcov[2][3];
      const double myBd3 = Bd3 + dqBd3 * di;
      const double ftemp = (1.0 - gcon03 * gcov03 - gcon13 * gcov13 - gcon23 * gcov23);
      const double igd = copysign(1.0, ftemp) / (fabs(ftemp) + O_SMALL);
      p[HARM_B3] = (myBd3 * gcon33 + Bu1 * gcon03 * gcov01 + Bu2 * gcon03 * gcov02 + Bu1 * gcon13 * gcov11 +
                    Bu2 * gcon13 * gcov12 + Bu1 * gcon23 * gcov21 + Bu2 * gcon23 * gcov22) * igd;
    }
    for (int pl = 0; pl < HARM_NPR; pl++) *cellp(o, P, pl, i, j, k) = p[pl];
  }
}

static void bound_x1(const orc *o, double *P, int nb) {
  const harm_grid *g = &o->g;
#pragma omp parallel for collapse(2) num_threads(o->nthreads)
  for (int k = 0; k < g->n3; k++)
    for (int j = 0; j < g->n2; j++) extrap_line(o, P, j, k, 0, 1, 2, 1.0, -nb, -1);
#pragma omp parallel for collapse(2) num_threads(o->nthreads)
  for (int k = 0; k < g->n3; k++)
    for (int j = 0; j < g->n2; j++) {
      const int ri = g->n1 - 1;
      extrap_line(o, P, j, k, ri, ri - 1, ri - 2, -1.0, ri + 1, ri + nb);
      for (int i = ri + 1; i <= ri + nb; i++) {
        ogeom gi;
        cent(o, i, j, &gi);
        double p[HARM_NPR];
        for (int pl = 0; pl < HARM_NPR; pl++) p[pl] = *cellp(o, P, pl, i, j, k);
        o_inflow_check_x1up(p, &gi, g->gammamax);
        o_limit_gamma(g->gammamax, p, &gi);
        for (int pl = 0; pl < HARM_NPR; pl++) *cellp(o, P, pl, i, j, k) = p[pl];
      }
    }
}

/* poledeath (bounds.tools.c:2004) at one pole for the column (i,k): the ghost cell and the
   first active cell next to the pole take rho, u, U1, U3 (and B3 in 2-D) of the second
   active cell rj; U2 there is the second cell's extrapolated linearly to zero at the pole,
   or zero where it flows into the pole; then POLEGAMMADEATH limits the Lorentz factor of
   the two cells (GAMMAPOLEOUTGOING 1.1 (r/10 beyond r = 10) where u^r > 0, else GAMMAMAX). */
static void poledeath_column(const orc *o, double *P, int i, int k, int up) {
  const harm_grid *g = &o->g;
  const int n2 = g->n2;
  const int rj = up ? n2 - 2 : 1;
  const int js = up ? n2 - 1 : -1, je = up ? n2 : 0;
  const int poleloc = up ? n2 : 0;
  const double Xr2 = x2c(g, rj), X02 = x2f(g, poleloc);
  for (int j = js; j <= je; j++) {
    for (int pl = HARM_RHO; pl <= HARM_U3; pl++) {
      if (pl == HARM_U2) continue;
      *cellp(o, P, pl, i, j, k) = *cellp(o, P, pl, i, rj, k);
    }
    double ftemp = *cellp(o, P, HARM_U2, i, rj, k);
    const double X2 = x2c(g, j);
    if ((!up && ftemp > 0.0) || (up && ftemp < 0.0)) ftemp = 0.0;
    *cellp(o, P, HARM_U2, i, j, k) = ftemp + (X2 - Xr2) * (ftemp - 0.0) / (Xr2 - X02);
    if (g->n3 == 1) *cellp(o, P, HARM_B3, i, j, k) = *cellp(o, P, HARM_B3, i, rj, k);
  }
}

static void polegamma_column(const orc *o, double *P, int i, int k, int up) {
  const harm_grid *g = &o->g;
  const int js = up ? g->n2 - 1 : -1, je = up ? g->n2 : 0;
  for (int j = js; j <= je; j++) {
    ogeom gi;
    cent(o, i, j, &gi);
    double p[HARM_NPR], ucon[4], gam, qsq;
    for (int pl = 0; pl < HARM_NPR; pl++) p[pl] = *cellp(o, P, pl, i, j, k);
    o_ucon(p, &gi, ucon, &gam, &qsq);
    if (ucon[1] > 0.0) {
      const double r = o->aux[(size_t)HARM_AUX_R * o->plane + (size_t)(j + g->ng) * g->n1e + (i + g->ng)];
      const double lim = (r <= 10.0) ? 1.1 : 1.1 * pow(r / 10.0, 1.0);
      o_limit_gamma(lim, p, &gi);
    } else {
      o_limit_gamma(g->gammamax, p, &gi);
    }
    for (int pl = 0; pl < HARM_NPR; pl++) *cellp(o, P, pl, i, j, k) = p[pl];
  }
}

static void bound_x2(const orc *o, double *P, int nb1, int nb) {
  const harm_grid *g = &o->g;
  const int n2 = g->n2, n3 = g->n3;
  for (int up = 0; up <= 1; up++) {
#pragma omp parallel for collapse(2) num_threads(o->nthreads)
    for (int k = 0; k < n3; k++)
      for (int i = -nb1; i < g->n1 + nb1; i++) {
        const int rk = k;
        for (int t = 1; t <= nb; t++) {
          const int j = up ? n2 - 1 + t : -t;
          const int rj = up ? 2 * (n2 - 1) - j + 1 : -j - 1;
          for (int pl = 0; pl < HARM_NPR; pl++) {
            double v = *cellp(o, P, pl, i, rj, rk);
            if (pl == HARM_U2 || pl == HARM_B2) v *= -1.;
            *cellp(o, P, pl, i, j, k) = v;
          }
        }
      }
#pragma omp parallel for collapse(2) num_threads(o->nthreads)
    for (int k = 0; k < n3; k++)
      for (int i = -nb1; i < g->n1 + nb1; i++) poledeath_column(o, P, i, k, up);
#pragma omp parallel for collapse(2) num_threads(o->nthreads)
    for (int k = 0; k < n3; k++)
      for (int i = -nb1; i < g->n1 + nb1; i++) polegamma_column(o, P, i, k, up);
  }
}

static void bound_x3(const orc *o, double *P, int nb1, int nb2, int nb) {
  const harm_grid *g = &o->g;
  const int n3 = g->n3;
#pragma omp parallel for collapse(2) num_threads(o->nthreads)
  for (int j = -nb2; j < g->n2 + nb2; j++)
    for (int i = -nb1; i < g->n1 + nb1; i++) {
      for (int t = 1; t <= nb; t++) {
        for (int pl = 0; pl < HARM_NPR; pl++) {
          *cellp(o, P, pl, i, j, -t) = *cellp(o, P, pl, i, j, n3 - t);
          *cellp(o, P, pl, i, j, n3 - 1 + t) = *cellp(o, P, pl, i, j, t - 1);
        }
      }
    }
}

/* one direction of bound_prim; simple = one ghost layer (BOUNDPRIMSIMPLETYPE) */
int orc_bound_dir(orc *o, double *P, int dir, int simple) {
  const harm_grid *g = &o->g;
  const int nb = simple ? 1 : g->ng, nb3 = (g->n3 > 1) ? (simple ? 1 : g->ng3) : 0;
  if (dir == 1) bound_x1(o, P, nb);
  else if (dir == 2) bound_x2(o, P, nb, nb);
  else if (dir == 3 && g->n3 > 1) bound_x3(o, P, nb, nb, nb3);
  return 0;
}

int orc_bound(orc *o, double *P) {
  for (int dir = 1; dir <= 3; dir++) orc_bound_dir(o, P, dir, 0);
  return 0;
}
