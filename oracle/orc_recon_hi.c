/*
 * orc_recon_hi.c -- TEST INFRASTRUCTURE ONLY (CPU oracle; see harm_oracle.h).
 * Higher-order line reconstructions (PPM para4, WENO5BND).
 */
#include "harm_oracle.h"
#include "orc_internal.h"

void o_recon_line_para(int n, const double *y, double *yl, double *yr) {
  for (int c = 0; c < n; c++) yl[c] = yr[c] = y[c];
}

void o_recon_line_weno5(int n, const double *y, double *yl, double *yr) {
  for (int c = 0; c < n; c++) yl[c] = yr[c] = y[c];
}
