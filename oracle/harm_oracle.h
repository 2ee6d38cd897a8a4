/*
 * harm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement (plain C, FP64, OpenMP) of HARM's per-timestep GRMHD update, used as
 * the checker of the device path in tests/, in __graft_entry__.smoke() and as the
 * timed CPU baseline of bench.py.  Nothing in the product library links or calls it.
 *
 * Parity status: the reference needs generated headers (decs.h from makedecs.h.sh,
 * global.defnprs.h from generatenprs.c) and its own build system, so it is not built
 * here; the reference's tests hold no golden vectors for this path.  Parity of this
 * oracle with the reference is therefore UNPINNED: each function cites the reference
 * file:line it restates, and tests/test_oracle_*.py check it against physics
 * known-answer properties (P->U->P round trips, free-stream fluxes, div B) instead.
 *
 * Every array is in the layout of include/harm_b200.h (SoA over the extended grid).
 */
#ifndef HARM_ORACLE_H
#define HARM_ORACLE_H
#include <stdint.h>
#include <stddef.h>
#include "harm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc {
  harm_grid g;
  const double *geom, *conn, *aux;
  size_t plane, cells;
  int nthreads;
} orc;

void orc_init(orc *o, const harm_grid *g, const double *geom, const double *conn,
              const double *aux, int nthreads);

/* single-point routines (geomrec = one CENT record of HARM_NGF doubles) */
void orc_primtoU_point(const double *geomrec, const double *pr, double *U);
void orc_primtoflux_point(const double *geomrec, const double *pr, int dir, double *F);
int orc_utoprimgen_point(const harm_grid *g, const double *geomrec, const double *U,
                         double *pr, int8_t *pflag, int32_t *iters);
void orc_vchar_point(const harm_grid *g, const double *geomrec, const double *pr, int dir,
                     double *vmax, double *vmin);

/* grid routines */
int orc_bound(orc *o, double *P);
int orc_bound_dir(orc *o, double *P, int dir, int simple);
int orc_fluxcalc(orc *o, const double *pb, double *F1, double *F2, double *F3, double ndt[3]);
int orc_advance(orc *o, int timeorder, int numtimeorders, const double *pi, const double *pb,
                double *pf, int8_t *pflag, double dt, const double CUf[4],
                const double Cunew[4], double *ndt, harm_stats *st);
int orc_advance_u(orc *o, int timeorder, int numtimeorders, const double *pi, const double *pb, double *pf,
                  int8_t *pflag, double *ui, double *uf, double *ucum, double dt, const double CUf[4],
                  const double Cunew[4], double *ndt, harm_stats *st);
int orc_post_fixup(orc *o, double *pf, int8_t *pflag, int finalstep);
int orc_step(orc *o, double *P, double *dt, harm_stats *st);

/* reconstruction of one line (tests): y[n] -> left/right edge values of each cell whose
   stencil fits (lim = PARALINE here without flattening) */
void orc_reconstruct_line(int lim, int n, const double *y, double *pl, double *pr);
/* PARALINE with the flattening of V[n] (sqrt(-g) rho u^dir) and P[n] (total pressure) */
void orc_paraline_flattener(int n, const double *V, const double *P, double *Fi);
void orc_reconstruct_line_paraline(int n, const double *y, const double *V, const double *P, double *pl,
                                   double *pr);
/* the PARALINE flattening coefficients fluxcalc uses on the line along dir through the
   transverse active-relative indices (a, b); Fi has the line's extended length */
void orc_paraline_line_fi(const orc *o, const double *pb, int dir, int a, int b, double *Fi);
/* the WENO5 momentum-flux jump indicator fluxcalc uses on the same line */
void orc_weno_line_dp(const orc *o, const double *pb, int dir, int a, int b, double *dP);

/* the 52 columns of one row of the main dump file (dump_content, dump.c:449) for active cell
   (i, j, k); U may be NULL (primtoU of P) */
void orc_dump_row(const orc *o, const double *P, const double *U, int i, int j, int k, double *out);

/* learned-guess network oracle (double precision; same parameter layout as the device) */
int orc_mlp_nparams(void);
void orc_mlp_features(const harm_grid *g, const double *geomrec, const double *U,
                      const double *P, float *feat, float *targ);
double orc_mlp_loss_grad(int n, const float *feat, const float *targ, const float *params,
                         const float *norm, double *pred, double *grad);

#ifdef __cplusplus
}
#endif
#endif
