/*
 * orc_advance.c -- TEST INFRASTRUCTURE ONLY (CPU oracle; see harm_oracle.h).
 *
 * advance_standard (advance.c:140) for one RK substep, post_fixup/fixup_utoprim
 * (fixup.c:53, :1061, general_average :1830) with the flags' ghost zones, and the full RK2 step
 * (step_ch_simplempi step_ch.c:524, setup_rktimestep :1244-1266, post_stepch :150).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "harm_oracle.h"
#include "orc_internal.h"

void orc_init(orc *o, const harm_grid *g, const double *geom, const double *conn,
              const double *aux, int nthreads) {
  o->g = *g;
  o->geom = geom;
  o->conn = conn;
  o->aux = aux;
  o->plane = (size_t)g->n1e * g->n2e;
  o->cells = o->plane * g->n3e;
  o->nthreads = nthreads > 0 ? nthreads : 1;
}

/* Ghost-zone flags for post_fixup's neighbour test: bound_pflag_user (boundsint.c:18) with the
   torus boundaries, in its order: x3 periodic over the full i, j extent first (so ghost cells
   in x1 or x2 of the x3 ghost planes take the values their periodic partners hold from the
   previous call), then the x1 outer OUTFLOW copy of the last active cell over the active j, k
   (the x1 inner boundary is FREEOUTFLOW, which bound_pflag_user leaves alone), then the x2
   POLARAXIS mirror within the same k plane over the full i extent and the active k. */
static void bound_flags(orc *o, int8_t *flag) {
  const harm_grid *g = &o->g;
  const int n1e = g->n1e, n2e = g->n2e, ng = g->ng, ng3 = g->ng3, n3 = g->n3;
  if (n3 > 1)
    for (int jj = 0; jj < n2e; jj++)
      for (int ii = 0; ii < n1e; ii++) {
        for (int kk = 0; kk < ng3; kk++) flag[oidx(o, ii, jj, kk)] = flag[oidx(o, ii, jj, kk + n3)];
        for (int kk = ng3 + n3; kk < g->n3e; kk++) flag[oidx(o, ii, jj, kk)] = flag[oidx(o, ii, jj, kk - n3)];
      }
  for (int kk = ng3; kk < ng3 + n3; kk++)
    for (int jj = ng; jj < ng + g->n2; jj++)
      for (int ii = ng + g->n1; ii < n1e; ii++) flag[oidx(o, ii, jj, kk)] = flag[oidx(o, ng + g->n1 - 1, jj, kk)];
  for (int kk = ng3; kk < ng3 + n3; kk++)
    for (int ii = 0; ii < n1e; ii++) {
      for (int jj = 0; jj < ng; jj++) flag[oidx(o, ii, jj, kk)] = flag[oidx(o, ii, 2 * ng - 1 - jj, kk)];
      for (int jj = ng + g->n2; jj < n2e; jj++) flag[oidx(o, ii, jj, kk)] = flag[oidx(o, ii, 2 * (ng + g->n2) - 1 - jj, kk)];
    }
}


int orc_advance(orc *o, int timeorder, int numtimeorders, const double *pi, const double *pb,
                double *pf, int8_t *pflag, double dt, const double CUf[4],
                const double Cunew[4], double *ndt, harm_stats *st) {
  return orc_advance_u(o, timeorder, numtimeorders, pi, pb, pf, pflag, NULL, NULL, NULL, dt, CUf, Cunew, ndt, st);
}

/* advance_standard (advance.c:140) with the conserved arrays of the RK step: ui = primtoU(pi)
   (advance.c:454), uf and ucum zeroed on the first substep (:407), then per cell dUtoU
   (advance.c:2046): uf = UFSET(CUf, dt, ui, uf, dUriemann, dUgeom), ucum += UCUMUPDATE(Cunew,
   dt, ui, uf, dUriemann, dUgeom) (global.stepch.h:1, :10), and the inversion of ucum on the
   final substep, of uf before (:671-679).  ui, uf, ucum NULL: the substep's uf and ucum start
   from zero (exact for TIMEORDER 1 and the RK2 midpoint, whose coefficients never carry them
   across substeps). */
int orc_advance_u(orc *o, int timeorder, int numtimeorders, const double *pi, const double *pb, double *pf,
                  int8_t *pflag, double *ui, double *uf, double *ucum, double dt, const double CUf[4],
                  const double Cunew[4], double *ndt, harm_stats *st) {
  const harm_grid *g = &o->g;
  const size_t cells = o->cells, plane = o->plane;
  const int finalstep = (timeorder == numtimeorders - 1);
  double *F1 = (double *)calloc(HARM_NPR * cells, sizeof(double));
  double *F2 = (double *)calloc(HARM_NPR * cells, sizeof(double));
  double *F3 = (double *)calloc(HARM_NPR * cells, sizeof(double));
  double *Uinv = (double *)calloc(HARM_NPR * cells, sizeof(double));
  double ndt3[3];
  orc_fluxcalc(o, pb, F1, F2, F3, ndt3);
  const int ng = g->ng, ng3 = g->ng3, has3 = g->n3 > 1;
  const double idx1 = 1.0 / g->dx[1], idx2 = 1.0 / g->dx[2], idx3 = 1.0 / g->dx[3];
  /* update loop (advance.c:420-575) */
#pragma omp parallel for collapse(2) schedule(static) num_threads(o->nthreads)
  for (int k = 0; k < g->n3; k++)
    for (int j = 0; j < g->n2; j++)
      for (int i = 0; i < g->n1; i++) {
        int ii = i + ng, jj = j + ng, kk = k + ng3;
        size_t id = oidx(o, ii, jj, kk);
        ogeom gc;
        og_load(o, HARM_LOC_CENT, ii, jj, &gc);
        double pri[HARM_NPR], prb[HARM_NPR], Ui[HARM_NPR], dUg[HARM_NPR];
        for (int p = 0; p < HARM_NPR; p++) { pri[p] = pi[p * cells + id]; prb[p] = pb[p * cells + id]; }
        ostate qi, qb;
        o_get_state(pri, &gc, g->gam, &qi);
        o_primtoflux(pri, &qi, 0, &gc, Ui);
        double dU[HARM_NPR];
        size_t ip = oidx(o, ii + 1, jj, kk), jp = oidx(o, ii, jj + 1, kk), kp = has3 ? oidx(o, ii, jj, kk + 1) : id;
        for (int p = 0; p < HARM_NPR; p++) {
          double d1 = -(F1[p * cells + ip] - F1[p * cells + id]) * idx1;
          double d2 = -(F2[p * cells + jp] - F2[p * cells + id]) * idx2;
          double d3 = has3 ? -(F3[p * cells + kp] - F3[p * cells + id]) * idx3 : 0.0;
          dU[p] = d1 + d2 + d3;
        }
        double conn[64];
        for (int c = 0; c < 64; c++) conn[c] = o->conn[(size_t)c * plane + (size_t)jj * g->n1e + ii];
        o_get_state(prb, &gc, g->gam, &qb);
        o_source(prb, &qb, &gc, conn, dUg);
        for (int p = 0; p < HARM_NPR; p++) {
          /* UFSET / UCUMUPDATE (global.stepch.h:1, :10) */
          const size_t q = p * cells + id;
          const double ufo = (uf && timeorder > 0) ? uf[q] : 0.0;
          const double uco = (ucum && timeorder > 0) ? ucum[q] : 0.0;
          double Uf = CUf[0] * Ui[p] + CUf[1] * ufo + CUf[2] * dt * (dU[p] + dUg[p]);
          double uc = uco + (Cunew[0] * Ui[p] + Cunew[1] * dt * (dU[p] + dUg[p]) + Cunew[2] * Uf);
          if (ui) ui[q] = Ui[p];
          if (uf) uf[q] = Uf;
          if (ucum) ucum[q] = uc;
          Uinv[q] = finalstep ? uc : Uf;
        }
      }
  /* pf = pb everywhere (copy_3dnpr_fullloop advance.c:654), then invert active cells */
  for (size_t c = 0; c < HARM_NPR * cells; c++) pf[c] = pb[c];
  double iters = 0.0, fails = 0.0, floors = 0.0;
#pragma omp parallel for collapse(2) schedule(dynamic, 4) reduction(+ : iters, fails, floors) num_threads(o->nthreads)
  for (int k = 0; k < g->n3; k++)
    for (int j = 0; j < g->n2; j++)
      for (int i = 0; i < g->n1; i++) {
        int ii = i + ng, jj = j + ng, kk = k + ng3;
        size_t id = oidx(o, ii, jj, kk);
        ogeom gc;
        og_load(o, HARM_LOC_CENT, ii, jj, &gc);
        double U[HARM_NPR], pr[HARM_NPR];
        for (int p = 0; p < HARM_NPR; p++) { U[p] = Uinv[p * cells + id]; pr[p] = pf[p * cells + id]; }
        int8_t fl = 0;
        int nst = 0;
        o_utoprimgen(U, &gc, pr, &fl, g->gam, g->gammafail, &nst);
        if (fl > 0) fails += 1.0;
        size_t c2 = (size_t)jj * g->n1e + ii;
        floors += o_fixup1zone(pr, &gc, o->aux[HARM_AUX_RHOFLOOR * plane + c2], o->aux[HARM_AUX_UFLOOR * plane + c2],
                               g->gam, g->gammamax, g->gammafail, &fl, &nst);
        iters += nst;
        pflag[id] = fl;
        for (int p = 0; p < HARM_NPR; p++) pf[p * cells + id] = pr[p];
      }
  /* prepare_globaldt (advance.c:1558), accdt = BIG (LIMITDTWITHSOURCETERM=0) */
  double wavedt = 1. / (1. / ndt3[0] + 1. / ndt3[1] + 1. / ndt3[2]);
  *ndt = g->defcon * fmin(wavedt, 1.e100);
  if (st) {
    st->newton_iters += iters;
    st->cells_inverted += (double)g->n1 * g->n2 * g->n3;
    st->inversion_failures += fails;
    st->floor_hits += floors;
  }
  free(F1); free(F2); free(F3); free(Uinv);
  return 0;
}

/* fixup_utoprim (fixup.c:1061) of post_fixup (fixup.c:53) with the torus configuration:
   UTOPRIMADJUST=UTOPRIMAVG, GENERALAVERAGE, CAUSALAVG=0, HOWTOAVG_WHEN_U2AVG=MAXUPOSAVG,
   HANDLE*NEG=0, DO_CONSERVE_D_INFAILFIXUPS=0, TODONOGOOD=NOGOODAVERAGE, USERRESETREGION=1
   (initboundcode/init.fishmon.h), WHICHPTOUSEWHENNOGOOD=0, STEPOVERNEG*=NEVERFIXUP.
   Per failed active cell (flag > 0), from the values before any fix (ptoavg):
   - which primitives: u alone for U2AVG1/U2AVG2/UPERC, else rho .. u^3 (fixup.c:1196-1218);
   - general_average (fixup.c:1830): the mean of the unfailed neighbours of the 3x3(x3) box
     summed in pairs, or for U2AVG the smallest u of the pairs whose both members are at
     least the cell's u;
   - no usable neighbour (fixup_nogood fixup.c:2291; never for U2AVG2): the mean of the 8
     in-plane neighbours (AVG4_1, AVG4_2 fixup.c:1812), failed or not, of those primitives;
     in the reset region (first 10 radial cells, two cells at either pole) rho and u are
     averaged so and the velocity set to the normal observer (zero ũ);
   - a fixed velocity has its Lorentz factor limited to the cell's own before the fix
     (at most GAMMAMAX);
   - fixuputoprim_accounting (fixup.c:1592): the flag becomes UTOPRIMFAILFIXEDUTOPRIM (-1),
     for the negative-density/energy and U2AVG codes only on the final substep. */
int orc_post_fixup(orc *o, double *pf, int8_t *pflag, int finalstep) {
  const harm_grid *g = &o->g;
  const size_t cells = o->cells;
  bound_flags(o, pflag);
  double *ptoavg = (double *)malloc(HARM_NPR * cells * sizeof(double));
  int8_t *forig = (int8_t *)malloc(cells);
  memcpy(ptoavg, pf, HARM_NPR * cells * sizeof(double));
  memcpy(forig, pflag, cells);
  const int s1 = g->n1 > 1, s2 = g->n2 > 1, s3 = g->n3 > 1;
  const int rnx = s1 ? 3 : 1, rny = s2 ? 3 : 1;
  const int npairs = ((int)pow(3, s1 + s2 + s3) - 1) / 2;
#pragma omp parallel for collapse(2) schedule(static) num_threads(o->nthreads)
  for (int k = 0; k < g->n3; k++)
    for (int j = 0; j < g->n2; j++)
      for (int i = 0; i < g->n1; i++) {
        int ii = i + g->ng, jj = j + g->ng, kk = k + g->ng3;
        size_t id = oidx(o, ii, jj, kk);
        int8_t f = forig[id];
        if (f <= 0) continue;
        const int u2 = (f == HARM_UTOPRIMFAILU2AVG1 || f == HARM_UTOPRIMFAILU2AVG2);
        int startpl, endpl;
        if (u2 || f == 13) {
          startpl = endpl = HARM_UU;
        } else {
          startpl = HARM_RHO;
          endpl = HARM_U3;
        }
        const int looptype = u2 ? 1 : 0;
        double mysum[2][HARM_NPR] = {{0}}, lastmin[HARM_NPR];
        for (int p = 0; p < HARM_NPR; p++) lastmin[p] = 1E50;
        int numavg0 = 0, numavg1 = 0;
        double ref = ptoavg[HARM_UU * cells + id];
        for (int qq = 0; qq < npairs; qq++) {
          int di = (qq % rnx) - s1, dj = ((qq % (rnx * rny)) / rnx) - s2, dk = (qq / (rnx * rny)) - s3;
          size_t a = oidx(o, ii + di, jj + dj, kk + dk), b = oidx(o, ii - di, jj - dj, kk - dk);
          int thisok = forig[a] <= 0, thatok = forig[b] <= 0;
          numavg0 += thisok + thatok;
          for (int p = startpl; p <= endpl; p++) {
            if (looptype == 0) {
              mysum[qq % 2][p] += ptoavg[p * cells + a] * thisok + ptoavg[p * cells + b] * thatok;
            } else {
              double f1 = ptoavg[p * cells + a], f2 = ptoavg[p * cells + b];
              if (f1 >= ref && f2 >= ref) {
                lastmin[p] = fmin(fmin(lastmin[p], f1), f2);
                numavg1++;
              }
            }
          }
        }
        int numavg;
        if (looptype == 0) {
          if (numavg0 != 0)
            for (int p = startpl; p <= endpl; p++) pf[p * cells + id] = (mysum[0][p] + mysum[1][p]) / (double)numavg0;
          numavg = numavg0;
        } else {
          if (numavg1 != 0)
            for (int p = startpl; p <= endpl; p++) pf[p * cells + id] = lastmin[p];
          numavg = numavg1;
        }
        if (f == HARM_UTOPRIMFAILU2AVG2) numavg++;
        if (numavg == 0) {
          /* fixup_nogood: 0.5 (AVG4_1 + AVG4_2) of ptoavg in the cell's k plane */
          const size_t ijp = oidx(o, ii, jj + 1, kk), ijm = oidx(o, ii, jj - 1, kk);
          const size_t imj = oidx(o, ii - 1, jj, kk), ipj = oidx(o, ii + 1, jj, kk);
          const size_t pp = oidx(o, ii + 1, jj + 1, kk), pm = oidx(o, ii + 1, jj - 1, kk);
          const size_t mp = oidx(o, ii - 1, jj + 1, kk), mm = oidx(o, ii - 1, jj - 1, kk);
          const int reset = (j <= 1 || j >= g->n2 - 2) || (i < 10);
          const int lo = reset ? HARM_RHO : startpl, hi = reset ? HARM_UU : endpl;
          for (int p = lo; p <= hi; p++) {
            const double *q = ptoavg + p * cells;
            double a4 = 0.25 * ((q[ijp] + q[ijm]) + (q[imj] + q[ipj]));
            double b4 = 0.25 * ((q[pp] + q[pm]) + (q[mp] + q[mm]));
            pf[p * cells + id] = 0.5 * (a4 + b4);
          }
          if (reset)
            for (int p = HARM_U1; p <= HARM_U3; p++) pf[p * cells + id] = 0.0;
        }
        if (startpl <= HARM_U1 && endpl >= HARM_U3) {
          ogeom gc;
          og_load(o, HARM_LOC_CENT, ii, jj, &gc);
          double pa[HARM_NPR], pv[HARM_NPR], ucon[4], gamma, qsq;
          for (int p = 0; p < HARM_NPR; p++) { pa[p] = ptoavg[p * cells + id]; pv[p] = pf[p * cells + id]; }
          o_ucon(pa, &gc, ucon, &gamma, &qsq);
          if (gamma > g->gammamax) gamma = g->gammamax;
          o_limit_gamma(gamma, pv, &gc);
          for (int p = 0; p < HARM_NPR; p++) pf[p * cells + id] = pv[p];
        }
        const int soft = (f == HARM_UTOPRIMFAILRHONEG || f == HARM_UTOPRIMFAILUNEG || f == HARM_UTOPRIMFAILRHOUNEG ||
                          u2);
        if (!soft || finalstep) pflag[id] = HARM_UTOPRIMFAILFIXEDUTOPRIM;
      }
  free(ptoavg);
  free(forig);
  return 0;
}

/* One RK2 midpoint step (TIMEORDER=2): CUf = {1,0,1/2},{1,0,1}; Cunew = {0,0,0},{0,0,1} */
int orc_step(orc *o, double *P, double *dt, harm_stats *st) {
  const size_t n = HARM_NPR * o->cells;
  double *pk = (double *)malloc(n * sizeof(double));
  int8_t *pflag = (int8_t *)calloc(o->cells, 1);
  const double CUf[2][4] = {{1.0, 0.0, 0.5, 0.0}, {1.0, 0.0, 1.0, 0.0}};
  const double Cun[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 1.0, 0.5}};
  double ndt, lastndt = 1.e100;
  /* substep 0: pi=P, pb=P, pf=pk */
  orc_advance(o, 0, 2, P, P, pk, pflag, *dt, CUf[0], Cun[0], &ndt, st);
  if (ndt < lastndt) lastndt = ndt;
  orc_bound(o, pk);
  orc_post_fixup(o, pk, pflag, 0);
  orc_bound(o, pk);
  /* substep 1: pi=P, pb=pk, pf=P */
  orc_advance(o, 1, 2, P, pk, P, pflag, *dt, CUf[1], Cun[1], &ndt, st);
  if (ndt < lastndt) lastndt = ndt;
  orc_bound(o, P);
  orc_post_fixup(o, P, pflag, 1);
  orc_bound(o, P);
  /* post_stepch (step_ch.c:213) */
  if (lastndt > o->g.safe * (*dt)) lastndt = o->g.safe * (*dt);
  *dt = lastndt;
  free(pk);
  free(pflag);
  return 0;
}
