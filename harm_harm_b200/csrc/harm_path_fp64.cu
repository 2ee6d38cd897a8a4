// harm_path_fp64.cu -- FP64 path of the step (compiled with -fmad=false) and the FP64
// kernels shared by both paths: boundary conditions, fixups, dt finalisation, point
// inversions.
//
// harm_path_fp64fma.cu compiles this file's flux and update launchers a second time, with
// FMA contraction and the inversion's shared reciprocals (HARM_FP64_FMA_TU): the FP64 path as
// fast as the compiler makes it, for comparisons of speed (HARM_PREC_FP64_FMA); this build
// (HARM_PREC_FP64) performs the CPU restatement's IEEE operations in its order.
// FP64 flux tiles at 2 resident blocks per SM (128 registers; harm_common.cuh): left to
// itself the compiler can take ~160 registers and 1 block per SM, which halves the resident
// warps (40.1 ms of flux per substep at 384x192x128 instead of 24.6)
#ifndef HARM_FLUXT_MINB
#define HARM_FLUXT_MINB 2
#endif
#include <algorithm>
#include "harm_common.cuh"
#include "harm_mlp_tc.cuh"
#include "harm_paths.h"

#ifdef HARM_FP64_FMA_TU
#define FP64_PATH 2
#define FP64_FN(name) name##fma
#else
#define FP64_PATH 0
#define FP64_FN(name) name
#endif

#ifndef HARM_FP64_FMA_TU

// copy p_b into the ghost zones of p_f (advance.c:654 copies the full grid)
__global__ void k_copy_ghosts(Dims d, const double* __restrict__ pb, double* __restrict__ pf) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)d.cells) return;
  int ii = (int)(t % d.n1e);
  long long r = t / d.n1e;
  int jj = (int)(r % d.n2e), kk = (int)(r / d.n2e);
  bool active = ii >= d.ng && ii < d.ng + d.n1 && jj >= d.ng && jj < d.ng + d.n2 && kk >= d.ng3 && kk < d.ng3 + d.n3;
  if (active) return;
#pragma unroll
  for (int p = 0; p < NPR; p++) pf[(size_t)p * d.cells + t] = pb[(size_t)p * d.cells + t];
}

// ------------------------------------------------------------------ boundary conditions
//
// bound_prim of the torus problem (step_ch.c:1332 -> bound_prim_user_dir,
// initboundcode/bounds.fishmon.c:15), direction by direction as bound_anyprim does:
//   x1: extrapfunc (bounds.tools.c:1417; HORIZONEXTRAP = OUTEREXTRAP = 3) fills the ghost
//       cells of each active (j,k) line from its three cells next to the boundary; at the
//       outer boundary inflow_check_rel4vel and limit_gamma follow (bound_x1up_outflow :337);
//   x2: polar reflection in the same phi plane with U2, B2 negated (bound_x2dn_polaraxis :751;
//       a run without MPI has periodicx3 = 0 and so no transfer across the pole), then
//       poledeath (:2004) on the ghost cell and the first active cell at each pole
//       (POLEDEATH 1, POLEINTERPTYPE 3) and POLEGAMMADEATH's Lorentz-factor limit there,
//       over every i of the extended grid;
//   x3: periodic (:1114), over every (i,j) of the extended grid.
// One thread per boundary line; the arithmetic is the oracle's (oracle/orc_bound.c) in the
// same order.

#define BMINMOD(a, b) (((a) * (b) <= 0) ? 0.0 : ((fabs(a) < fabs(b)) ? (a) : (b)))

__device__ __forceinline__ void cent_geo(const Dims& d, const double* __restrict__ geom, int ii, int jj,
                                         Geo<double>& g) {
  load_geo<double, double>(geom + (size_t)HARM_LOC_CENT * HARM_NGF * d.plane, d.plane, (size_t)jj * d.n1e + ii, g);
}

// extrapfunc for the ghost cells of the x1 line (jj,kk) on one side
__global__ void k_bound_x1_extrap(Dims d, Phys ph, double* __restrict__ P, const double* __restrict__ geom) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2LL * d.n2 * d.n3) return;
  const int up = (int)(t & 1);
  long long r = t >> 1;
  const int jj = (int)(r % d.n2) + d.ng, kk = (int)(r / d.n2) + d.ng3;
  const int ri = up ? d.ng + d.n1 - 1 : d.ng;
  const int ri2 = up ? ri - 1 : ri + 1, ri3 = up ? ri - 2 : ri + 2;
  const double signdq = up ? -1.0 : 1.0;
  Geo<double> gr, g2, g3;
  cent_geo(d, geom, ri, jj, gr);
  cent_geo(d, geom, ri2, jj, g2);
  cent_geo(d, geom, ri3, jj, g3);
  double p1[NPR], p2[NPR], p3[NPR];
  const size_t c1 = cidx(d, ri, jj, kk), c2 = cidx(d, ri2, jj, kk), c3 = cidx(d, ri3, jj, kk);
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) {
    p1[pl] = P[(size_t)pl * d.cells + c1];
    p2[pl] = P[(size_t)pl * d.cells + c2];
    p3[pl] = P[(size_t)pl * d.cells + c3];
  }
  double Bd3 = 0.0, Bd3ri2 = 0.0, Bd3ri3 = 0.0;
  for (int a = 1; a <= 3; a++) Bd3 += p1[HARM_B1 + a - 1] * gr.gcov[sym(3, a)];
  for (int a = 1; a <= 3; a++) Bd3ri2 += p2[HARM_B1 + a - 1] * g2.gcov[sym(3, a)];
  for (int a = 1; a <= 3; a++) Bd3ri3 += p3[HARM_B1 + a - 1] * g3.gcov[sym(3, a)];
  double Dqp = Bd3ri3 - Bd3ri2, Dqm = Bd3ri2 - Bd3, Dqc = Bd3ri3 - Bd3;
  const double dqBd3 = signdq * BMINMOD(BMINMOD(Dqp, Dqm), Dqc);
  double ucref[4], ucref2[4], gam, qsq;
  ucon_of<double>(p1, gr, ucref, gam, qsq);
  ucon_of<double>(p2, g2, ucref2, gam, qsq);
  double dq[NPR], dqlog[NPR], dqgd[NPR];
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) {
    Dqp = p3[pl] - p2[pl];
    Dqm = p2[pl] - p1[pl];
    Dqc = p3[pl] - p1[pl];
    dq[pl] = signdq * BMINMOD(BMINMOD(Dqp, Dqm), Dqc);
    Dqp = log(1.e-300 + fabs(p3[pl])) - log(1.e-300 + fabs(p2[pl]));
    Dqm = log(1.e-300 + fabs(p2[pl])) - log(1.e-300 + fabs(p1[pl]));
    Dqc = log(1.e-300 + fabs(p3[pl])) - log(1.e-300 + fabs(p1[pl]));
    dqlog[pl] = signdq * BMINMOD(BMINMOD(Dqp, Dqm), Dqc);
    Dqp = g3.gdet * p3[pl] - g2.gdet * p2[pl];
    Dqm = g2.gdet * p2[pl] - gr.gdet * p1[pl];
    Dqc = g3.gdet * p3[pl] - gr.gdet * p1[pl];
    dqgd[pl] = signdq * BMINMOD(BMINMOD(Dqp, Dqm), Dqc);
  }
  // the slopes of u and the velocities fade out where u^t jumps between ri and ri2
  const double xdqfrac = fabs(ucref[0] - ucref2[0]) / ucref[0];
  double ydqfrac;
  if (xdqfrac < 0.1) ydqfrac = 0.0;
  else if (xdqfrac < 0.2) ydqfrac = (0.0 + (1.0 - 0.0) / (0.2 - 0.1) * (xdqfrac - 0.1));
  else ydqfrac = 1.0;
#pragma unroll
  for (int a = 0; a < 4; a++) {
    dq[HARM_UU + a] = dq[HARM_UU + a] * (1.0 - ydqfrac);
    dqlog[HARM_UU + a] = dqlog[HARM_UU + a] * (1.0 - ydqfrac);
  }
  const double powerratio = (1.0 + (0.1));
  for (int q = 1; q <= d.ng; q++) {
    const int ii = up ? ri + q : ri - q;
    const double di = (double)(ii - ri);
    Geo<double> gi;
    cent_geo(d, geom, ii, jj, gi);
    double p[NPR];
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) p[pl] = p1[pl];
#pragma unroll
    for (int pl = HARM_RHO; pl <= HARM_UU; pl++) {
      double ftemp = exp(-signdq * dqlog[pl]) - powerratio, mydqlog;
      if (ftemp >= 0.0) mydqlog = log(powerratio) / (-signdq);
      else mydqlog = dqlog[pl];
      p[pl] = exp(log(1.e-300 + fabs(p1[pl])) + mydqlog * di);
    }
#pragma unroll
    for (int pl = HARM_U1; pl <= HARM_U3; pl++) p[pl] = p1[pl] + dq[pl] * di;
#pragma unroll
    for (int pl = HARM_B1; pl <= HARM_B2; pl++) {
      const double igd = copysign(1.0, gi.gdet) / (fabs(gi.gdet) + 1.e-300);
      p[pl] = (p1[pl] * fabs(gr.gdet + dqgd[pl] * di)) * igd;
    }
    {
      const double Bu1 = p[HARM_B1], Bu2 = p[HARM_B2];
      const double gcon03 = gi.gcon[sym(0, 3)], gcon13 = gi.gcon[sym(1, 3)], gcon23 = gi.gcon[sym(2, 3)],
                   gcon33 = gi.gcon[sym(3, 3)];
      const double gcov01 = gi.gcov[sym(0, 1)], gcov02 = gi.gcov[sym(0, 2)], gcov11 = gi.gcov[sym(1, 1)],
                   gcov12 = gi.gcov[sym(1, 2)], gcov21 = gcov12, gcov22 = gi.gcov[sym(2, 2)],
                   gcov03 = gi.gcov[sym(0, 3)], gcov13 = gi.gcov[sym(1, 3)], gcov23 = gi.gcov[sym(2, 3)];
      const double myBd3 = Bd3 + dqBd3 * di;
      const double ftemp = (1.0 - gcon03 * gcov03 - gcon13 * gcov13 - gcon23 * gcov23);
      const double igd = copysign(1.0, ftemp) / (fabs(ftemp) + 1.e-300);
      p[HARM_B3] = (myBd3 * gcon33 + Bu1 * gcon03 * gcov01 + Bu2 * gcon03 * gcov02 + Bu1 * gcon13 * gcov11 +
                    Bu2 * gcon13 * gcov12 + Bu1 * gcon23 * gcov21 + Bu2 * gcon23 * gcov22) * igd;
    }
    if (up) {
      // inflow_check_rel4vel (fixup.c:3255) for the outer radial boundary, then limit_gamma
      double ucon[4], gamma, qsq2;
      ucon_of<double>(p, gi, ucon, gamma, qsq2);
      if (ucon[1] < 0.) {
        p[HARM_U1] /= gamma; p[HARM_U2] /= gamma; p[HARM_U3] /= gamma;
        double alpha = 1. / sqrt(-gi.gcon[0]);
        double betacon = gi.gcon[1] * alpha * alpha;
        p[HARM_U1] = betacon / alpha;
        double vsq = 0.;
        for (int a = 1; a < 4; a++)
          for (int b = 1; b < 4; b++) vsq += gi.gcov[sym(a, b)] * p[HARM_U1 + a - 1] * p[HARM_U1 + b - 1];
        if (vsq < 0.0 && vsq > -2.220446049250313e-16 * 100.0) vsq = 0.0;
        if (vsq >= 1.0) vsq = 1.0 - 1.0 / (ph.gammamax * ph.gammamax);
        gamma = 1. / sqrt(1. - vsq);
        p[HARM_U1] *= gamma; p[HARM_U2] *= gamma; p[HARM_U3] *= gamma;
      }
      limit_gamma<double>(ph.gammamax, p, gi);
    }
    const size_t c = cidx(d, ii, jj, kk);
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) P[(size_t)pl * d.cells + c] = p[pl];
  }
}

// polar reflection of the ghost rows of column (ii,kk) at both poles
__global__ void k_bound_x2_reflect(Dims d, double* __restrict__ P) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2LL * d.n1e * d.n3) return;
  const int up = (int)(t & 1);
  long long r = t >> 1;
  const int ii = (int)(r % d.n1e), kk = (int)(r / d.n1e) + d.ng3;
  for (int q = 1; q <= d.ng; q++) {
    const int j = up ? d.n2 - 1 + q : -q;
    const int rj = up ? 2 * (d.n2 - 1) - j + 1 : -j - 1;
    const size_t dst = cidx(d, ii, j + d.ng, kk), src = cidx(d, ii, rj + d.ng, kk);
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) {
      double v = P[(size_t)pl * d.cells + src];
      if (pl == HARM_U2 || pl == HARM_B2) v *= -1.;
      P[(size_t)pl * d.cells + dst] = v;
    }
  }
}

// poledeath and POLEGAMMADEATH of column (ii,kk) at one pole: the ghost cell and the first
// active cell take rho, u, U1, U3 (and B3 in 2-D) of the second active cell; U2 there is the
// second cell's extrapolated linearly to zero at the pole, or zero where it flows into the
// pole; then the Lorentz factor is limited (1.1, growing as r/10 beyond r = 10, where u^r > 0;
// GAMMAMAX otherwise)
__global__ void k_bound_x2_pole(Dims d, Phys ph, double startx2, double* __restrict__ P,
                                const double* __restrict__ geom, const double* __restrict__ aux) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2LL * d.n1e * d.n3) return;
  const int up = (int)(t & 1);
  long long r = t >> 1;
  const int ii = (int)(r % d.n1e), kk = (int)(r / d.n1e) + d.ng3;
  const int rj = up ? d.n2 - 2 : 1, js = up ? d.n2 - 1 : -1, poleloc = up ? d.n2 : 0;
  const double Xr2 = startx2 + (rj + 0 + 0.5) * ph.dx2, X02 = startx2 + (poleloc + 0) * ph.dx2;
  const size_t cr = cidx(d, ii, rj + d.ng, kk);
  for (int j = js; j <= js + 1; j++) {
    const size_t c = cidx(d, ii, j + d.ng, kk);
#pragma unroll
    for (int pl = HARM_RHO; pl <= HARM_U3; pl++) {
      if (pl == HARM_U2) continue;
      P[(size_t)pl * d.cells + c] = P[(size_t)pl * d.cells + cr];
    }
    double ftemp = P[(size_t)HARM_U2 * d.cells + cr];
    const double X2 = startx2 + (j + 0 + 0.5) * ph.dx2;
    if ((!up && ftemp > 0.0) || (up && ftemp < 0.0)) ftemp = 0.0;
    P[(size_t)HARM_U2 * d.cells + c] = ftemp + (X2 - Xr2) * (ftemp - 0.0) / (Xr2 - X02);
    if (d.n3 == 1) P[(size_t)HARM_B3 * d.cells + c] = P[(size_t)HARM_B3 * d.cells + cr];
  }
  for (int j = js; j <= js + 1; j++) {
    const int jj = j + d.ng;
    const size_t c = cidx(d, ii, jj, kk);
    Geo<double> gi;
    cent_geo(d, geom, ii, jj, gi);
    double p[NPR], ucon[4], gamma, qsq;
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) p[pl] = P[(size_t)pl * d.cells + c];
    ucon_of<double>(p, gi, ucon, gamma, qsq);
    if (ucon[1] > 0.0) {
      const double rr = aux[(size_t)HARM_AUX_R * d.plane + (size_t)jj * d.n1e + ii];
      const double lim = (rr <= 10.0) ? 1.1 : 1.1 * pow(rr / 10.0, 1.0);
      limit_gamma<double>(lim, p, gi);
    } else {
      limit_gamma<double>(ph.gammamax, p, gi);
    }
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) P[(size_t)pl * d.cells + c] = p[pl];
  }
}

__global__ void k_bound_x3(Dims d, double* P, int8_t* flag) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)2 * d.ng3 * d.plane;
  if (t >= n) return;
  int ii = (int)(t % d.n1e);
  long long r = t / d.n1e;
  int jj = (int)(r % d.n2e), gq = (int)(r / d.n2e);
  int kk, ks;
  if (gq < d.ng3) { kk = gq; ks = kk + d.n3; }
  else { kk = d.ng3 + d.n3 + (gq - d.ng3); ks = kk - d.n3; }
  size_t dst = cidx(d, ii, jj, kk), src = cidx(d, ii, jj, ks);
  if (flag) flag[dst] = flag[src];
  if (P)
    for (int p = 0; p < NPR; p++) P[(size_t)p * d.cells + dst] = P[(size_t)p * d.cells + src];
}

// Ghost flags for post_fixup's neighbour test, as bound_pflag_user (boundsint.c:18) sets
// them for the torus, in its order: x3 periodic first over the full i, j extent (k_bound_x3;
// ghost cells in x1 or x2 of the x3 ghost planes so take the values their periodic partners
// hold from the previous call), then the x1 outer OUTFLOW copy of the last active cell over
// the active j, k (k_bound_flags_x1; the inner x1 boundary is FREEOUTFLOW, which leaves its
// ghost flags alone), then the x2 POLARAXIS mirror within the same k plane over the full i
// extent and the active k (k_bound_flags_x2).
__global__ void k_bound_flags_x1(Dims d, int8_t* flag) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)d.ng * d.n2 * d.n3;
  if (t >= n) return;
  int gq = (int)(t % d.ng);
  long long r = t / d.ng;
  int jj = (int)(r % d.n2) + d.ng, kk = (int)(r / d.n2) + d.ng3;
  int ii = d.ng + d.n1 + gq;
  flag[cidx(d, ii, jj, kk)] = flag[cidx(d, d.ng + d.n1 - 1, jj, kk)];
}

__global__ void k_bound_flags_x2(Dims d, int8_t* flag) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)2 * d.ng * d.n1e * d.n3;
  if (t >= n) return;
  int ii = (int)(t % d.n1e);
  long long r = t / d.n1e;
  int gq = (int)(r % (2 * d.ng)), kk = (int)(r / (2 * d.ng)) + d.ng3;
  int jj, js;
  if (gq < d.ng) { jj = gq; js = 2 * d.ng - 1 - jj; }
  else { jj = d.ng + d.n2 + (gq - d.ng); js = 2 * (d.ng + d.n2) - 1 - jj; }
  flag[cidx(d, ii, jj, kk)] = flag[cidx(d, ii, js, kk)];
}

// ------------------------------------------------------------------ post_fixup


// fixup_utoprim (fixup.c:1061) of post_fixup (fixup.c:53), the torus configuration: per failed
// active cell, from the values before any fix, the primitives to fix (u alone for
// U2AVG1/U2AVG2/UPERC, else rho .. u^3), general_average (fixup.c:1830: the mean of the unfailed
// neighbours of the 3x3(x3) box summed in pairs, or for U2AVG the smallest u of the pairs
// whose both members are at least the cell's), where no neighbour is usable fixup_nogood
// (fixup.c:2291: the mean of the 8 in-plane neighbours, failed or not; in the reset region of
// USERRESETREGION, the first 10 radial cells and two cells at either pole, rho and u so and
// a zero velocity), the Lorentz-factor limit of a fixed velocity to the cell's own (at most
// GAMMAMAX), and the flag of fixuputoprim_accounting (fixup.c:1592): -1, for the negative
// density/energy and U2AVG codes only on the final substep.  Each fixed cell is recorded and
// written by k_fixup_apply, so that every cell's fix reads the unfixed neighbours.
__global__ void __launch_bounds__(256) k_fixup_compute(Dims d, Phys ph, const double* __restrict__ P,
                                                       const int8_t* __restrict__ flag, const double* __restrict__ geom,
                                                       FixRec* __restrict__ recs, unsigned int* __restrict__ nrec,
                                                       unsigned int cap, int finalstep) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)d.n1 * d.n2 * d.n3) return;
  int i = (int)(t % d.n1);
  long long r = t / d.n1;
  int j = (int)(r % d.n2), k = (int)(r / d.n2);
  int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
  size_t id = cidx(d, ii, jj, kk);
  int8_t f = flag[id];
  if (f <= 0) return;
  int startpl, endpl;
  const bool u2 = (f == HARM_UTOPRIMFAILU2AVG1 || f == HARM_UTOPRIMFAILU2AVG2);
  if (u2 || f == 13) { startpl = endpl = HARM_UU; }
  else { startpl = HARM_RHO; endpl = HARM_U3; }
  const int s1 = d.n1 > 1, s2 = d.n2 > 1, s3 = d.n3 > 1;
  const int rnx = s1 ? 3 : 1, rny = s2 ? 3 : 1;
  const int npairs = ((s1 + s2 + s3) == 3 ? 27 : (s1 + s2 + s3) == 2 ? 9 : 3) / 2;
  double sum0[5] = {0, 0, 0, 0, 0}, sum1[5] = {0, 0, 0, 0, 0}, lastmin[5];
  for (int p = 0; p < 5; p++) lastmin[p] = 1E50;
  int numavg0 = 0, numavg1 = 0;
  const double ref = P[(size_t)HARM_UU * d.cells + id];
  for (int qq = 0; qq < npairs; qq++) {
    int di = (qq % rnx) - s1, dj = ((qq % (rnx * rny)) / rnx) - s2, dk = (qq / (rnx * rny)) - s3;
    size_t a = cidx(d, ii + di, jj + dj, kk + dk), b = cidx(d, ii - di, jj - dj, kk - dk);
    int thisok = flag[a] <= 0, thatok = flag[b] <= 0;
    numavg0 += thisok + thatok;
    for (int p = startpl; p <= endpl; p++) {
      double fa = P[(size_t)p * d.cells + a], fb = P[(size_t)p * d.cells + b];
      if (!u2) {
        double add = fa * thisok + fb * thatok;
        if (qq % 2 == 0) sum0[p] += add; else sum1[p] += add;
      } else if (fa >= ref && fb >= ref) {
        lastmin[p] = fmin(fmin(lastmin[p], fa), fb);
        numavg1++;
      }
    }
  }
  double out[5];
  for (int p = 0; p < 5; p++) out[p] = P[(size_t)p * d.cells + id];
  int numavg;
  if (!u2) {
    if (numavg0 != 0)
      for (int p = startpl; p <= endpl; p++) out[p] = (sum0[p] + sum1[p]) / (double)numavg0;
    numavg = numavg0;
  } else {
    if (numavg1 != 0)
      for (int p = startpl; p <= endpl; p++) out[p] = lastmin[p];
    numavg = numavg1;
  }
  if (f == HARM_UTOPRIMFAILU2AVG2) numavg++;
  if (numavg == 0) {  // fixup_nogood: 0.5 (AVG4_1 + AVG4_2) in the cell's k plane
    const bool reset = (j <= 1 || j >= d.n2 - 2) || (i < 10);
    const int lo = reset ? HARM_RHO : startpl, hi = reset ? HARM_UU : endpl;
    for (int p = lo; p <= hi; p++) {
      const double* q = P + (size_t)p * d.cells;
      const double a4 = 0.25 * ((q[cidx(d, ii, jj + 1, kk)] + q[cidx(d, ii, jj - 1, kk)]) +
                                (q[cidx(d, ii - 1, jj, kk)] + q[cidx(d, ii + 1, jj, kk)]));
      const double b4 = 0.25 * ((q[cidx(d, ii + 1, jj + 1, kk)] + q[cidx(d, ii + 1, jj - 1, kk)]) +
                                (q[cidx(d, ii - 1, jj + 1, kk)] + q[cidx(d, ii - 1, jj - 1, kk)]));
      out[p] = 0.5 * (a4 + b4);
    }
    if (reset)
      for (int p = HARM_U1; p <= HARM_U3; p++) out[p] = 0.0;
  }
  if (startpl <= HARM_U1 && endpl >= HARM_U3) {
    Geo<double> g;
    load_geo<double, double>(geom, d.plane, (size_t)jj * d.n1e + ii, g);
    double pa[NPR], pv[NPR];
    for (int p = 0; p < NPR; p++) pa[p] = P[(size_t)p * d.cells + id];
    for (int p = 0; p < NPR; p++) pv[p] = (p < 5) ? out[p] : pa[p];
    double ucon[4], gamma, qsq;
    ucon_of<double>(pa, g, ucon, gamma, qsq);
    if (gamma > ph.gammamax) gamma = ph.gammamax;
    limit_gamma<double>(gamma, pv, g);
    for (int p = 0; p < 5; p++) out[p] = pv[p];
  }
  const bool soft = (f == HARM_UTOPRIMFAILRHONEG || f == HARM_UTOPRIMFAILUNEG || f == HARM_UTOPRIMFAILRHOUNEG || u2);
  unsigned int slot = atomicAdd(nrec, 1u);
  if (slot < cap) {
    recs[slot].id = (long long)id;
    for (int p = 0; p < 5; p++) recs[slot].v[p] = out[p];
    recs[slot].flag = (!soft || finalstep) ? HARM_UTOPRIMFAILFIXEDUTOPRIM : f;
  }
}

__global__ void k_fixup_apply(Dims d, double* __restrict__ P, int8_t* __restrict__ flag,
                              const FixRec* __restrict__ recs, const unsigned int* __restrict__ nrec, unsigned int cap) {
  unsigned int n = *nrec;
  if (n > cap) n = cap;
  for (unsigned int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    size_t id = (size_t)recs[s].id;
    for (int p = 0; p < 5; p++) P[(size_t)p * d.cells + id] = recs[s].v[p];
    flag[id] = (int8_t)recs[s].flag;
  }
}

// ------------------------------------------------------------------ dt

// slots[6]: per substep s (0,1) and direction d the atomic min of cour dx/ctop.
__global__ void k_finalize_dt(Phys ph, unsigned long long* slots, double* dt, double* ndt_out, int nsub) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double last = 1.e100;
  for (int s = 0; s < nsub; s++) {
    double nd[3];
    for (int q = 0; q < 3; q++) {
      unsigned long long b = slots[s * 3 + q];
      nd[q] = (b == 0xFFFFFFFFFFFFFFFFull) ? 1.e100 : __longlong_as_double((long long)b);
    }
    double wavedt = 1. / (1. / nd[0] + 1. / nd[1] + 1. / nd[2]);
    double ndt = ph.defcon * fmin(wavedt, 1.e100);
    if (ndt_out) ndt_out[s] = ndt;
    if (ndt < last) last = ndt;
  }
  if (dt) {
    double cur = *dt;
    if (last > ph.safe * cur) last = ph.safe * cur;
    *dt = last;
  }
  for (int q = 0; q < 3 * nsub; q++) slots[q] = 0xFFFFFFFFFFFFFFFFull;
}

// ------------------------------------------------------------------ points inversion

__global__ void k_utoprim_points(size_t n, Phys ph, const double* __restrict__ U, const double* __restrict__ geom,
                                 double* __restrict__ P, int8_t* __restrict__ pflag, int32_t* __restrict__ iters) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  Geo<double> g;
  load_geo<double, double>(geom, n, t, g);
  double u[NPR], pr[NPR];
  for (int p = 0; p < NPR; p++) { u[p] = U[(size_t)p * n + t]; pr[p] = P[(size_t)p * n + t]; }
  int8_t flag = 0;
  int it = utoprimgen(u, g, g.igdet, pr, flag, ph.gam, ph.gammafail, false, 0.0, nullptr);
  for (int p = 0; p < NPR; p++) P[(size_t)p * n + t] = pr[p];
  pflag[t] = flag;
  if (iters) iters[t] = it;
}

// the same with the learned start of the hot inversion (fallback to the plain start inside
// utoprimgen); stats[2] counts the fallbacks
__global__ void __launch_bounds__(256, 2) k_utoprim_points_mlp(size_t n, Phys ph, const double* __restrict__ U,
                                                               const double* __restrict__ geom, double* __restrict__ P,
                                                               int8_t* __restrict__ pflag, int32_t* __restrict__ iters,
                                                               const MlpPacked* __restrict__ mlp, double* stats) {
  __shared__ MlpPacked sm;
  __shared__ MlpWarpScratch wsc[8];
  mlp_load_packed(sm, mlp);
  __syncthreads();
  double fb_d = 0.0;
  for (size_t base = (size_t)blockIdx.x * 256; base < n; base += (size_t)gridDim.x * 256) {
    const size_t t = base + threadIdx.x;
    const bool valid = t < n;
    Geo<double> g;
    double u[NPR], pr[NPR];
    float f[MLP_IN];
    JonSetup s;
    if (valid) {
      load_geo<double, double>(geom, n, t, g);
      double Ugf[NPR], prc[NPR];
      for (int p = 0; p < NPR; p++) {
        u[p] = U[(size_t)p * n + t];
        pr[p] = P[(size_t)p * n + t];
        Ugf[p] = u[p] * g.igdet;
        prc[p] = pr[p];
      }
      jon_prepare(false, Ugf, g, prc, ph.gam, ph.gammafail, s);
      mlp_features(s.c, g, f);
    }
    float y[MLP_OUT];
    mlp_warp_eval(sm, wsc[threadIdx.x >> 5], f, valid, y);
    if (valid) {
      int8_t flag = 0;
      bool failed = false;
      int it = utoprimgen(u, g, g.igdet, pr, flag, ph.gam, ph.gammafail, true, mlp_wp_guess(y[0], sm.start_bias, s),
                          &failed);
      fb_d += failed ? 1.0 : 0.0;
      for (int p = 0; p < NPR; p++) P[(size_t)p * n + t] = pr[p];
      pflag[t] = flag;
      if (iters) iters[t] = it;
    }
  }
  if (stats) warp_add_atomic(fb_d, stats + 2);
}

#endif  // HARM_FP64_FMA_TU

// ------------------------------------------------------------------ launchers

template <int LIM>
static int flux_dirs_double(harm_ctx* c, const Dims& d, const Phys& ph, const double* pb, double* F1, double* F2, double* F3,
                         unsigned long long* slots, const SlabWait* sw) {
  // WENO5: the cell pass computes the dP line quantities once per cell for the three directions
  double* L = (LIM == HARM_LIM_WENO5) ? reinterpret_cast<double*>(c->d_line) : nullptr;
  if (sw) {
    CK((launch_flux_slabs<LIM, double, double>(d, ph, pb, c->d_geom, F1, F2, F3, slots, c->stream, *sw, c->launches, L)));
    return 0;
  }
  if (L) {
    CK((launch_cellprep<double, double>(d, ph, pb, c->d_geom, L, 0, d.n3e, c->stream)));
    c->launches++;
  }
  FaceBox b1 = face_box(d, 1), b2 = face_box(d, 2), b3 = face_box(d, 3);
  CK((launch_fluxt<1, LIM, double, double>(d, ph, b1, pb, c->d_geom, F1, slots + 0, c->stream, L)));
  CK((launch_fluxt<2, LIM, double, double>(d, ph, b2, pb, c->d_geom, F2, slots + 1, c->stream, L)));
  c->launches += 2;
  if (d.n3 > 1) {
    CK((launch_fluxt<3, LIM, double, double>(d, ph, b3, pb, c->d_geom, F3, slots + 2, c->stream, L)));
    c->launches++;
  }
  return 0;
}

int FP64_FN(hp_fluxes_fp64)(harm_ctx* c, const double* pb, double* F1, double* F2, double* F3, double* emf,
                            unsigned long long* slots, const SlabWait* sw) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  if (c->g.lim == HARM_LIM_WENO5) { int rc = flux_dirs_double<HARM_LIM_WENO5>(c, d, ph, pb, F1, F2, F3, slots, sw); if (rc) return rc; }
  else if (c->g.lim == HARM_LIM_PARA) { int rc = flux_dirs_double<HARM_LIM_PARA>(c, d, ph, pb, F1, F2, F3, slots, sw); if (rc) return rc; }
  else if (c->g.lim == HARM_LIM_PARALINE) { int rc = flux_dirs_double<HARM_LIM_PARALINE>(c, d, ph, pb, F1, F2, F3, slots, sw); if (rc) return rc; }
  else { int rc = flux_dirs_double<HARM_LIM_MC>(c, d, ph, pb, F1, F2, F3, slots, sw); if (rc) return rc; }
  long long nc = (long long)(d.n1 + 1) * (d.n2 + 1) * (d.n3 > 1 ? d.n3 + 1 : 1);
  k_emf<double, double><<<nblk(nc), 256, 0, c->stream>>>(d, F1, F2, F3, c->d_geom, emf);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

int FP64_FN(hp_update_fp64)(harm_ctx* c, const StepCoef& sc, const double* pi, const double* pb, double* pf,
                            int8_t* pflag, double* stats) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  const CellTile ct = cell_tile(d.n3, HARM_INVERT_LTK);
  const CellTile cct = (HARM_CONSERVED_LTK > 0 && d.n3 >= 8) ? cell_tile(d.n3, HARM_CONSERVED_LTK) : cell_linear();
  if (ct.lti == 4) {  // 16 i x 16 k tiles: the metric and connection staged per block
    k_conserved<double, true><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(
        d, ph, sc, c->d_dt, pi, pb, c->d_F[0], c->d_F[1], c->d_F[2], c->d_emf, c->d_geom, c->d_conn, c->d_U, ct);
  } else {
    k_conserved<double><<<cell_grid(d.n1, d.n2, d.n3, cct), 256, 0, c->stream>>>(d, ph, sc, c->d_dt, pi, pb, c->d_F[0], c->d_F[1],
                                                            c->d_F[2], c->d_emf, c->d_geom, c->d_conn, c->d_U, cct);
  }
  CK(cudaMemsetAsync(c->d_nrare, 0, sizeof(unsigned int), c->stream));
  if (sc.guess == HARM_GUESS_MLP && c->mlp_tc == 4) {
    if (int rc = launch_invert_gated<FP64_PATH>(c, d, ph, ct, pb, pf, pflag, stats)) return rc;
  } else if (sc.guess == HARM_GUESS_MLP && c->mlp_tc == 2) {
    if (int rc = launch_invert_tc<FP64_PATH>(c, d, ph, pb, pf, pflag, stats)) return rc;
  } else if (sc.guess == HARM_GUESS_MLP && c->mlp_tc == 3) {
    if (int rc = launch_invert_mma<FP64_PATH>(c, d, ph, ct, pb, pf, pflag, stats)) return rc;
  } else if (sc.guess == HARM_GUESS_MLP) {
    if (c->mlp_tc == 1) {
      if (int rc = launch_mlp_guess_tc<FP64_PATH>(c, d)) return rc;
    } else {
      k_mlp_guess<FP64_PATH><<<HARM_MLP_GUESS_BLOCKS * c->num_sms, 256, 0, c->stream>>>(d, c->d_U, c->d_geom, c->d_wpg,
                                                      reinterpret_cast<const MlpPacked*>(c->d_mlp), ct);
      c->launches++;
    }
    k_invert<FP64_PATH, true><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag,
                                                          c->d_geom, c->d_aux, c->d_rare, c->d_nrare, stats, ct, c->d_wpg);
    c->launches++;
  } else {
    k_invert<FP64_PATH><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag, c->d_geom,
                                                    c->d_aux, c->d_rare, c->d_nrare, stats, ct);
    c->launches++;
  }
  k_invert_rare<FP64_PATH><<<2 * c->num_sms, 128, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag, c->d_geom, c->d_aux, c->d_rare,
                                                     c->d_nrare, stats);
  c->launches += 2;
  CK(cudaGetLastError());
  return 0;
}

#ifndef HARM_FP64_FMA_TU
int hp_emf_to_flux_fp64(harm_ctx* c, const double* emf, double* F1, double* F2, double* F3) {
  Dims d = dims_of(c->g);
  long long nc = (long long)(d.n1 + 1) * (d.n2 + 1) * (d.n3 > 1 ? d.n3 + 1 : 1);
  k_emf_to_flux<double><<<nblk(nc), 256, 0, c->stream>>>(d, emf, F1, F2, F3);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

int hp_bound(harm_ctx* c, double* P, int8_t* flag) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  if (P) {
    k_bound_x1_extrap<<<nblk(2LL * d.n2 * d.n3, 128), 128, 0, c->stream>>>(d, ph, P, c->d_geom);
    k_bound_x2_reflect<<<nblk(2LL * d.n1e * d.n3, 128), 128, 0, c->stream>>>(d, P);
    k_bound_x2_pole<<<nblk(2LL * d.n1e * d.n3, 128), 128, 0, c->stream>>>(d, ph, c->g.startx[2], P, c->d_geom, c->d_aux);
    c->launches += 3;
    if (d.n3 > 1) {
      k_bound_x3<<<nblk(2LL * d.ng3 * (long long)d.plane), 256, 0, c->stream>>>(d, P, nullptr);
      c->launches++;
    }
  }
  if (flag) {
    if (d.n3 > 1) {
      k_bound_x3<<<nblk(2LL * d.ng3 * (long long)d.plane), 256, 0, c->stream>>>(d, nullptr, flag);
      c->launches++;
    }
    k_bound_flags_x1<<<nblk((long long)d.ng * d.n2 * d.n3), 256, 0, c->stream>>>(d, flag);
    k_bound_flags_x2<<<nblk(2LL * d.ng * d.n1e * d.n3), 256, 0, c->stream>>>(d, flag);
    c->launches += 2;
  }
  CK(cudaGetLastError());
  return 0;
}

int hp_copy_ghosts(harm_ctx* c, const double* pb, double* pf) {
  Dims d = dims_of(c->g);
  k_copy_ghosts<<<nblk((long long)d.cells), 256, 0, c->stream>>>(d, pb, pf);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

int hp_fixup(harm_ctx* c, double* pf, int8_t* pflag, int finalstep, bool bound_flags) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  if (bound_flags && hp_bound(c, nullptr, pflag)) return 1;
  CK(cudaMemsetAsync(c->d_nrec, 0, sizeof(unsigned int), c->stream));
  long long ncell = (long long)d.n1 * d.n2 * d.n3;
  k_fixup_compute<<<nblk(ncell), 256, 0, c->stream>>>(d, ph, pf, pflag, c->d_geom, (FixRec*)c->d_fixrec, c->d_nrec,
                                                       c->fix_cap, finalstep);
  k_fixup_apply<<<4 * c->num_sms, 256, 0, c->stream>>>(d, pf, pflag, (const FixRec*)c->d_fixrec, c->d_nrec, c->fix_cap);
  c->launches += 2;
  CK(cudaGetLastError());
  return 0;
}

int hp_finalize_dt(harm_ctx* c, double* dt, double* ndt_out, int nsub) {
  Phys ph = phys_of(c->g);
  k_finalize_dt<<<1, 32, 0, c->stream>>>(ph, c->d_dtslots, dt, ndt_out, nsub);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

int hp_points(harm_ctx* c, size_t n, int guess, const double* U, const double* geom, double* P, int8_t* pflag,
              int32_t* iters) {
  Phys ph = phys_of(c->g);
  if (guess == HARM_GUESS_MLP) {
    const unsigned int nb = (unsigned int)std::min<size_t>((n + 255) / 256, (size_t)2 * c->num_sms);
    k_utoprim_points_mlp<<<nb, 256, 0, c->stream>>>(n, ph, U, geom, P, pflag, iters,
                                                   reinterpret_cast<const MlpPacked*>(c->d_mlp), c->d_stats);
  } else {
    k_utoprim_points<<<nblk((long long)n), 256, 0, c->stream>>>(n, ph, U, geom, P, pflag, iters);
  }
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}
#endif  // HARM_FP64_FMA_TU
