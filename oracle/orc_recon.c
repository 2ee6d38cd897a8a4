/*
 * orc_recon.c -- TEST INFRASTRUCTURE ONLY (CPU oracle; see harm_oracle.h).
 *
 * Reconstruction of one line of cell-centred values y[0..n-1] into the left-edge value
 * yl[c] and right-edge value yr[c] of each cell c whose stencil fits in the line.  The
 * face between cells c-1 and c gets p_l = yr[c-1], p_r = yl[c] (getp2interplr,
 * flux.c:2115).
 *
 *   MC   : slope_lim_3points + get_limit_slopes (interppoint.c:753, :769):
 *          dq = MINMOD(dq2, MINMOD(2 dq1l, 2 dq1r)), edges y -/+ dq/2.
 *   PARA, WENO5, PARALINE: orc_recon_hi.c (PARALINE's flattening needs the whole primitive
 *          state of each cell and is applied by the flux loop, orc_flux.c).
 */
#include <math.h>
#include <string.h>
#include "harm_oracle.h"
#include "orc_internal.h"

#define MINMODB(a, b) ((fabs(a) < fabs(b)) ? (a) : (b))
#define MINMOD(a, b) (((a) * (b) <= 0) ? 0.0 : MINMODB(a, b))

static double mc_slope(double yl, double yc, double yr) {
  double dq1l = 1.0 * (yc - yl), dq1r = 1.0 * (yr - yc), dq2 = 0.5 * (yr - yl);
  double Dqm = 2.0 * dq1l, Dqp = 2.0 * dq1r, Dqc = dq2;
  return MINMOD(Dqc, MINMOD(Dqm, Dqp));
}

void o_recon_line_para(int n, const double *y, double *yl, double *yr);

void o_recon_line(int lim, int n, const double *y, double *yl, double *yr) {
  for (int c = 0; c < n; c++) yl[c] = yr[c] = y[c];
  if (lim == HARM_LIM_MC) {
    for (int c = 1; c < n - 1; c++) {
      double dq = mc_slope(y[c - 1], y[c], y[c + 1]);
      yl[c] = y[c] - 0.5 * dq;
      yr[c] = y[c] + 0.5 * dq;
    }
  } else if (lim == HARM_LIM_PARA) {
    o_recon_line_para(n, y, yl, yr);
  } else if (lim == HARM_LIM_PARALINE) {
    o_recon_line_paraline(n, y, NULL, yl, yr);
  } else {
    o_recon_line_weno5(n, y, NULL, yl, yr);
  }
}

void orc_reconstruct_line(int lim, int n, const double *y, double *pl, double *pr) {
  o_recon_line(lim, n, y, pl, pr);
}
