/*
 * orc_flux.c -- TEST INFRASTRUCTURE ONLY (CPU oracle; see harm_oracle.h).
 *
 * fluxcalc (flux.c:38) restated: per direction, line reconstruction of the primitives
 * (orc_recon.c; for PARALINE with the flattening coefficients of the line), face states with B^dir made continuous (getplpr flux.c:1952, BDIRCONT=1)
 * and limit_gamma on each side (check_plpr flux.c:2041, EVOLVECHECKS=1), fluid state and
 * fluxes of both sides (p2SFUevolve fluxcompute.c:122), vchar wave speeds and
 * cminmax_calc (wavespeeds.c:12, :397, ROEAVERAGEDWAVESPEED=0), the HLL flux with the
 * LAXF fallback (hllflux_compute fluxcompute.c:329) or, for fluxmethod LAXF, the LAXF flux
 * (fluxcompute.c:243), the CFL dt = cour dx/ctop
 * (flux.c:1106), then Toth's flux-CT (flux_ct fluxct.c:186, CORNGDETVERSION=1).
 *
 * Faces computed per direction d: the faces bounding active cells in d and one layer of
 * transverse ghost faces on each side (needed by the corner EMFs).  The field fluxes are
 * final only on the faces of active cells.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "harm_oracle.h"
#include "orc_internal.h"

static void face_loop_bounds(const orc *o, int dir, int lo[3], int hi[3]) {
  const harm_grid *g = &o->g;
  int n[3] = {g->n1, g->n2, g->n3};
  for (int d = 0; d < 3; d++) {
    if (d == dir - 1) { lo[d] = 0; hi[d] = n[d]; }
    else if (n[d] > 1) { lo[d] = -1; hi[d] = n[d]; }
    else { lo[d] = 0; hi[d] = 0; }
  }
}

/* flux of one face (flux_compute fluxcompute.c:212): fluxmethod HLLFLUX (HLLCOMPUTE :179, the
   LAXF formula where cmax + cmin = 0, hllflux_compute :329) or LAXFFLUX (LAXFCOMPUTE :182) */
static void face_flux(const orc *o, int dir, const ogeom *g, double *pl, double *pr, double *F, double *ctop) {
  const harm_grid *hg = &o->g;
  /* getplpr: B^dir continuous */
  int bp = HARM_B1 + dir - 1;
  pl[bp] = pr[bp] = 0.5 * (pl[bp] + pr[bp]);
  /* check_plpr: limit_gamma on both states */
  o_limit_gamma(hg->gammamax, pl, g);
  o_limit_gamma(hg->gammamax, pr, g);
  ostate ql, qr;
  double Fl[HARM_NPR], Fr[HARM_NPR], Ul[HARM_NPR], Ur[HARM_NPR];
  o_get_state(pl, g, hg->gam, &ql);
  o_get_state(pr, g, hg->gam, &qr);
  o_primtoflux(pl, &ql, dir, g, Fl);
  o_primtoflux(pl, &ql, 0, g, Ul);
  o_primtoflux(pr, &qr, dir, g, Fr);
  o_primtoflux(pr, &qr, 0, g, Ur);
  double cmaxl, cminl, cmaxr, cminr;
  o_vchar(pl, &ql, dir, g, hg->gam, &cmaxl, &cminl);
  o_vchar(pr, &qr, dir, g, hg->gam, &cmaxr, &cminr);
  double lmin = fmin(cminl, cminr), lmax = fmax(cmaxl, cmaxr);
  lmin = fabs(fmax(0., -lmin));
  lmax = fabs(fmax(0., lmax));
  double cmin = lmin, cmax = lmax;
  *ctop = fmax(lmax, lmin);
  if (hg->fluxmethod != HARM_FLUX_LAXF && cmax + cmin != 0.0) {
    for (int p = 0; p < HARM_NPR; p++)
      F[p] = ((cmax * Fl[p] + cmin * Fr[p]) - (cmax * cmin) * (Ur[p] - Ul[p])) / (cmax + cmin);
  } else {
    for (int p = 0; p < HARM_NPR; p++) F[p] = 0.5 * ((Fl[p] + Fr[p]) - *ctop * (Ur[p] - Ul[p]));
  }
}

/* PARALINE flattening coefficients of the line along dir through the transverse
   active-relative indices (a, b) (dir 1: (j, k), dir 2: (i, k), dir 3: (i, j)):
   get_V_and_P (interpline.c:2964) gives V = sqrt(-g) rho u^dir and P = p + b^2/2 of every cell
   of the line at the cell centre, then o_paraline_flattener */
static void paraline_line_fi(const orc *o, const double *pb, int dir, int a, int b, double *Fi) {
  const harm_grid *g = &o->g;
  const int ng = g->ng, ng3 = g->ng3;
  const int nline = (dir == 1) ? g->n1e : (dir == 2) ? g->n2e : g->n3e;
  double *V = (double *)malloc(sizeof(double) * nline), *Pt = (double *)malloc(sizeof(double) * nline);
  for (int s = 0; s < nline; s++) {
    int ii, jj, kk;
    if (dir == 1) { ii = s; jj = a + ng; kk = b + ng3; }
    else if (dir == 2) { ii = a + ng; jj = s; kk = b + ng3; }
    else { ii = a + ng; jj = b + ng; kk = s; }
    double pr[HARM_NPR];
    for (int p = 0; p < HARM_NPR; p++) pr[p] = pb[(size_t)p * o->cells + oidx(o, ii, jj, kk)];
    ogeom gc;
    og_load(o, HARM_LOC_CENT, ii, jj, &gc);
    ostate q;
    o_get_state(pr, &gc, g->gam, &q);
    V[s] = gc.gdet * pr[HARM_RHO] * q.ucon[dir];
    Pt[s] = q.pressure;
    Pt[s] += 0.5 * q.bsq;
  }
  o_paraline_flattener(nline, V, Pt, Fi);
  free(V);
  free(Pt);
}

void orc_paraline_line_fi(const orc *o, const double *pb, int dir, int a, int b, double *Fi) {
  paraline_line_fi(o, pb, dir, a, b, Fi);
}

/* WENO5BND: the momentum-flux jump indicator dP of every cell of the line along dir through
   (a, b) (get_df_line_gen_new interpline.c:1473 -> compute_df_line_new), from the cells'
   primitives and centre geometry */
static void weno_line_dp(const orc *o, const double *pb, int dir, int a, int b, double *dP) {
  const harm_grid *g = &o->g;
  const int ng = g->ng, ng3 = g->ng3;
  const int nline = (dir == 1) ? g->n1e : (dir == 2) ? g->n2e : g->n3e;
  double *pr = (double *)malloc(sizeof(double) * HARM_NPR * (size_t)nline);
  ogeom *gc = (ogeom *)malloc(sizeof(ogeom) * (size_t)nline);
  for (int s = 0; s < nline; s++) {
    int ii, jj, kk;
    if (dir == 1) { ii = s; jj = a + ng; kk = b + ng3; }
    else if (dir == 2) { ii = a + ng; jj = s; kk = b + ng3; }
    else { ii = a + ng; jj = b + ng; kk = s; }
    for (int p = 0; p < HARM_NPR; p++) pr[(size_t)p * nline + s] = pb[(size_t)p * o->cells + oidx(o, ii, jj, kk)];
    og_load(o, HARM_LOC_CENT, ii, jj, &gc[s]);
  }
  o_weno_dp_line(nline, dir, pr, gc, g->gam, dP);
  free(pr);
  free(gc);
}

void orc_weno_line_dp(const orc *o, const double *pb, int dir, int a, int b, double *dP) {
  weno_line_dp(o, pb, dir, a, b, dP);
}

int orc_fluxcalc(orc *o, const double *pb, double *F1, double *F2, double *F3, double ndt[3]) {
  const harm_grid *g = &o->g;
  const size_t cells = o->cells;
  double *Fs[4] = {NULL, F1, F2, F3};
  int nd[4] = {0, g->n1, g->n2, g->n3};
  for (int d = 1; d <= 3; d++) ndt[d - 1] = 1.e100; /* BIG */
  for (int dir = 1; dir <= 3; dir++) {
    if (nd[dir] <= 1) continue;
    int lo[3], hi[3];
    face_loop_bounds(o, dir, lo, hi);
    int loc = (dir == 1) ? HARM_LOC_FACE1 : (dir == 2) ? HARM_LOC_FACE2 : HARM_LOC_CENT;
    double dtmin = 1.e100;
    int ng = g->ng, ng3 = g->ng3;
    /* lines along dir: iterate over transverse indices */
    int ta = (dir == 1) ? 1 : 0, tb = (dir == 3) ? 1 : 2; /* transverse dims (0-based) */
    int nline = (dir == 1) ? g->n1e : (dir == 2) ? g->n2e : g->n3e;
#pragma omp parallel for collapse(2) reduction(min : dtmin) schedule(static) num_threads(o->nthreads)
    for (int b = lo[tb]; b <= hi[tb]; b++)
      for (int a = lo[ta]; a <= hi[ta]; a++) {
        double *y = (double *)malloc(sizeof(double) * nline);
        double *yl = (double *)malloc(sizeof(double) * nline * HARM_NPR);
        double *yr = (double *)malloc(sizeof(double) * nline * HARM_NPR);
        /* extended transverse indices */
        int e[3];
        double *Fi = NULL, *dP = NULL;
        if (g->lim == HARM_LIM_PARALINE) {
          Fi = (double *)malloc(sizeof(double) * nline);
          paraline_line_fi(o, pb, dir, a, b, Fi);
        } else if (g->lim == HARM_LIM_WENO5) {
          dP = (double *)malloc(sizeof(double) * nline);
          weno_line_dp(o, pb, dir, a, b, dP);
        }
        for (int p = 0; p < HARM_NPR; p++) {
          for (int s = 0; s < nline; s++) {
            int ii, jj, kk;
            if (dir == 1) { ii = s; jj = a + ng; kk = b + ng3; }
            else if (dir == 2) { ii = a + ng; jj = s; kk = b + ng3; }
            else { ii = a + ng; jj = b + ng; kk = s; }
            y[s] = pb[(size_t)p * cells + oidx(o, ii, jj, kk)];
          }
          if (Fi) o_recon_line_paraline(nline, y, Fi, yl + (size_t)p * nline, yr + (size_t)p * nline);
          else if (dP) o_recon_line_weno5(nline, y, dP, yl + (size_t)p * nline, yr + (size_t)p * nline);
          else o_recon_line(g->lim, nline, y, yl + (size_t)p * nline, yr + (size_t)p * nline);
        }
        free(Fi);
        free(dP);
        int off = (dir == 3) ? ng3 : ng;
        for (int f = lo[dir - 1]; f <= hi[dir - 1]; f++) {
          int s = f + off; /* extended index of the cell above the face */
          if (dir == 1) { e[0] = s; e[1] = a + ng; e[2] = b + ng3; }
          else if (dir == 2) { e[0] = a + ng; e[1] = s; e[2] = b + ng3; }
          else { e[0] = a + ng; e[1] = b + ng; e[2] = s; }
          double pl[HARM_NPR], pr[HARM_NPR], F[HARM_NPR], ctop;
          for (int p = 0; p < HARM_NPR; p++) {
            pl[p] = yr[(size_t)p * nline + s - 1];
            pr[p] = yl[(size_t)p * nline + s];
          }
          ogeom gf;
          og_load(o, loc, e[0], e[1], &gf);
          face_flux(o, dir, &gf, pl, pr, F, &ctop);
          size_t id = oidx(o, e[0], e[1], e[2]);
          for (int p = 0; p < HARM_NPR; p++) Fs[dir][(size_t)p * cells + id] = F[p];
          double dtij = g->cour * g->dx[dir] / ctop;
          if (dtij < dtmin) dtmin = dtij;
        }
        free(y); free(yl); free(yr);
      }
    ndt[dir - 1] = dtmin;
  }
  /* ------------------------------------------------------------ flux_ct (Toth) */
  const int n1 = g->n1, n2 = g->n2, n3 = g->n3, ng = g->ng, ng3 = g->ng3;
  const int has3 = (n3 > 1);
  double c1 = has3 ? 0.25 : 0.5, c2 = has3 ? 0.25 : 0.5, c3 = 0.25;
  double *emf = (double *)calloc(3 * cells, sizeof(double));
  const size_t plane = o->plane;
#define GD(loc, ii, jj) (o->geom[((size_t)(loc) * HARM_NGF + HARM_G_GDET) * plane + (size_t)(jj) * g->n1e + (ii)])
#define IG(loc, ii, jj) (o->geom[((size_t)(loc) * HARM_NGF + HARM_G_IGDET) * plane + (size_t)(jj) * g->n1e + (ii)])
#define FF(Fa, pl, ii, jj, kk) (Fa[(size_t)(pl) * cells + oidx(o, ii, jj, kk)])
  int klo = has3 ? 0 : 0, khi = has3 ? n3 : 0;
#pragma omp parallel for collapse(2) schedule(static) num_threads(o->nthreads)
  for (int k = klo; k <= khi; k++)
    for (int j = 0; j <= n2; j++)
      for (int i = 0; i <= n1; i++) {
        int ii = i + ng, jj = j + ng, kk = k + ng3;
        int km = has3 ? kk - 1 : kk;
        /* stripped field fluxes: F * igdet at the face of each flux */
        double f2b3 = FF(F2, HARM_B3, ii, jj, kk) * IG(HARM_LOC_FACE2, ii, jj);
        double f2b3m = FF(F2, HARM_B3, ii, jj, km) * IG(HARM_LOC_FACE2, ii, jj);
        double f1b3 = FF(F1, HARM_B3, ii, jj, kk) * IG(HARM_LOC_FACE1, ii, jj);
        double f1b3m = FF(F1, HARM_B3, ii, jj, km) * IG(HARM_LOC_FACE1, ii, jj);
        double f1b2 = FF(F1, HARM_B2, ii, jj, kk) * IG(HARM_LOC_FACE1, ii, jj);
        double f1b2m = FF(F1, HARM_B2, ii, jj - 1, kk) * IG(HARM_LOC_FACE1, ii, jj - 1);
        double f2b1 = FF(F2, HARM_B1, ii, jj, kk) * IG(HARM_LOC_FACE2, ii, jj);
        double f2b1m = FF(F2, HARM_B1, ii - 1, jj, kk) * IG(HARM_LOC_FACE2, ii - 1, jj);
        double e1, e2, e3;
        if (has3) {
          double f3b2 = FF(F3, HARM_B2, ii, jj, kk) * IG(HARM_LOC_CENT, ii, jj);
          double f3b2m = FF(F3, HARM_B2, ii, jj - 1, kk) * IG(HARM_LOC_CENT, ii, jj - 1);
          double f3b1 = FF(F3, HARM_B1, ii, jj, kk) * IG(HARM_LOC_CENT, ii, jj);
          double f3b1m = FF(F3, HARM_B1, ii - 1, jj, kk) * IG(HARM_LOC_CENT, ii - 1, jj);
          e1 = c1 * (+f2b3 + f2b3m - f3b2 - f3b2m);
          e2 = c2 * (+f3b1 + f3b1m - f1b3 - f1b3m);
        } else {
          e1 = c1 * (+f2b3 + f2b3m);
          e2 = c2 * (-f1b3 - f1b3m);
        }
        e3 = c3 * (+f1b2 + f1b2m - f2b1 - f2b1m);
        size_t id = oidx(o, ii, jj, kk);
        emf[0 * cells + id] = e1 * GD(HARM_LOC_FACE2, ii, jj); /* CORN1 shares FACE2 */
        emf[1 * cells + id] = e2 * GD(HARM_LOC_FACE1, ii, jj); /* CORN2 shares FACE1 */
        emf[2 * cells + id] = e3 * GD(HARM_LOC_CORN3, ii, jj);
      }
  /* EMF -> field fluxes on the faces of active cells (fluxct.c:1110-1160) */
#define EMF(c, ii, jj, kk) (emf[(size_t)(c) * cells + oidx(o, ii, jj, kk)])
#pragma omp parallel for collapse(2) schedule(static) num_threads(o->nthreads)
  for (int k = 0; k < n3; k++)
    for (int j = 0; j <= n2; j++)
      for (int i = 0; i <= n1; i++) {
        int ii = i + ng, jj = j + ng, kk = k + ng3;
        int kp = has3 ? kk + 1 : kk;
        if (j < n2) {
          FF(F1, HARM_B1, ii, jj, kk) = 0.;
          FF(F1, HARM_B2, ii, jj, kk) = 0.5 * (EMF(2, ii, jj, kk) + EMF(2, ii, jj + 1, kk));
          FF(F1, HARM_B3, ii, jj, kk) = -0.5 * (EMF(1, ii, jj, kk) + EMF(1, ii, jj, kp));
        }
        if (i < n1) {
          FF(F2, HARM_B1, ii, jj, kk) = -0.5 * (EMF(2, ii, jj, kk) + EMF(2, ii + 1, jj, kk));
          FF(F2, HARM_B2, ii, jj, kk) = 0.;
          FF(F2, HARM_B3, ii, jj, kk) = 0.5 * (EMF(0, ii, jj, kk) + EMF(0, ii, jj, kp));
        }
      }
  if (has3) {
#pragma omp parallel for collapse(2) schedule(static) num_threads(o->nthreads)
    for (int k = 0; k <= n3; k++)
      for (int j = 0; j < n2; j++)
        for (int i = 0; i < n1; i++) {
          int ii = i + ng, jj = j + ng, kk = k + ng3;
          FF(F3, HARM_B1, ii, jj, kk) = 0.5 * (EMF(1, ii, jj, kk) + EMF(1, ii + 1, jj, kk));
          FF(F3, HARM_B2, ii, jj, kk) = -0.5 * (EMF(0, ii, jj, kk) + EMF(0, ii, jj + 1, kk));
          FF(F3, HARM_B3, ii, jj, kk) = 0.;
        }
  }
  free(emf);
  return 0;
#undef GD
#undef IG
#undef FF
#undef EMF
}
