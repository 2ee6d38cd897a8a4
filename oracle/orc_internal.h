/* orc_internal.h -- TEST INFRASTRUCTURE ONLY: shared declarations of the CPU oracle. */
#ifndef ORC_INTERNAL_H
#define ORC_INTERNAL_H
#include "harm_oracle.h"

#define O_SMALL (1.e-300) /* SMALL for doubles (global.depnmemonics.h:493) */

typedef struct ogeom {
  double gcov[4][4], gcon[4][4];
  double gcovpert_tt, alpha, betasqoalphasq, beta[4], gdet, igdet;
} ogeom;

typedef struct ostate {
  double ucon[4], ucov[4], bsq, pressure, plus1ud0, gamma, qsq;
} ostate;

void og_from_record(const double *rec, ogeom *g);
void og_load(const orc *o, int loc, int ii, int jj, ogeom *g);
void o_lower(const double *ucon, const ogeom *g, double *ucov);
void o_raise(const double *ucov, const ogeom *g, double *ucon);
double o_qsq(const double *pr, const ogeom *g);
void o_ucon(const double *pr, const ogeom *g, double *ucon, double *gamma, double *qsq);
void o_get_state(const double *pr, const ogeom *g, double gam, ostate *q);
void o_primtoflux(const double *pr, const ostate *q, int dir, const ogeom *g, double *F);
int o_vchar(const double *pr, const ostate *q, int dir, const ogeom *g, double gam, double *vmax, double *vmin);
void o_source(const double *pr, const ostate *q, const ogeom *g, const double *conn, double *dU);
int o_utoprimgen(const double *U, const ogeom *g, double *pr, int8_t *pflag, double gam, double gammafail, int *nstroke);
void o_inv_invariants(const double *Ugf, const ogeom *g, double *out);
int o_limit_gamma(double gammamax, double *pr, const ogeom *g);
void o_inflow_check_x1up(double *pr, const ogeom *g, double gammamax);
int o_fixup1zone(double *pr, const ogeom *g, double rhofl, double ufl, double gam, double gammamax,
                 double gammafail, int8_t *pflag, int *nstroke);

/* reconstruction of a 1-D line of n values at n-? faces; see orc_recon.c */
void o_recon_line(int lim, int n, const double *y, double *yl, double *yr);
/* PARALINE: flattening coefficients of cells 3..n-4 from V, P (others 0), and the edges of a
   line with given coefficients (Fi NULL: none); see orc_recon_hi.c */
void o_paraline_flattener(int n, const double *V, const double *P, double *Fi);
void o_recon_line_paraline(int n, const double *y, const double *Fi, double *yl, double *yr);
/* WENO5BND with the momentum-flux jump indicator dP[n] of the line's cells (NULL: no
   reduction by it); see orc_recon_hi.c */
void o_recon_line_weno5(int n, const double *y, const double *dP, double *yl, double *yr);
/* dP of each cell of a line from the cells' primitives pr[p * n + s] and centre geometry */
void o_weno_dp_line(int n, int dir, const double *pr, const ogeom *g, double gam, double *dP);

static inline size_t oidx(const orc *o, int ii, int jj, int kk) {
  return ((size_t)kk * o->g.n2e + jj) * o->g.n1e + ii;
}
#endif
