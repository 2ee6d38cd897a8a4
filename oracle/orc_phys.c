/*
 * orc_phys.c -- TEST INFRASTRUCTURE ONLY (CPU oracle; see harm_oracle.h).
 *
 * Per-cell physics of HARM restated in C: the fluid state (get_state), fluxes and
 * conserved variables (primtoflux/primtoU), fast magnetosonic speeds (vchar/simplefast),
 * the connection source (source_conn), the Utoprimgen inversion with Jon's 1-D W'
 * Newton method and the cold fallback, limit_gamma, the inflow check and fixup1zone.
 * Configuration restated: WHICHVEL=VELREL4, REMOVERESTMASSFROMUU=2, MAXWELL=PRIMMAXWELL,
 * WHICHEOM=WITHGDET, ideal gas, UTOPRIMVERSION=UTOPRIMJONNONRELCOMPAT with
 * WHICHHOTINVERTER=3, WHICHCOLDINVERTER=2, PRECISEINVERSION=1, HOT2COLD=1,
 * HOT2ENTROPY=0 (NPR=8 carries no entropy), UTOPRIMFAILRETURNTYPE=ADJUSTED, FIXUPTYPE=1.
 */
#include <float.h>
#include <math.h>
#include <string.h>
#include "harm_oracle.h"
#include "orc_internal.h"

/* ---------------------------------------------------------------- geometry */

static const int SYM[4][4] = {{0, 1, 2, 3}, {1, 4, 5, 6}, {2, 5, 7, 8}, {3, 6, 8, 9}};

void og_from_record(const double *rec, ogeom *g) {
  for (int m = 0; m < 4; m++)
    for (int n = 0; n < 4; n++) {
      g->gcov[m][n] = rec[HARM_G_GCOV + SYM[m][n]];
      g->gcon[m][n] = rec[HARM_G_GCON + SYM[m][n]];
    }
  g->gcovpert_tt = rec[HARM_G_GCOVPERT_TT];
  g->alpha = rec[HARM_G_ALPHA];
  g->betasqoalphasq = rec[HARM_G_BETASQOALPHASQ];
  g->beta[0] = 0.0;
  for (int j = 1; j < 4; j++) g->beta[j] = rec[HARM_G_BETA + j - 1];
  g->gdet = rec[HARM_G_GDET];
  g->igdet = rec[HARM_G_IGDET];
}

void og_load(const orc *o, int loc, int ii, int jj, ogeom *g) {
  double rec[HARM_NGF];
  size_t c = (size_t)jj * o->g.n1e + ii;
  for (int f = 0; f < HARM_NGF; f++) rec[f] = o->geom[((size_t)loc * HARM_NGF + f) * o->plane + c];
  og_from_record(rec, g);
}

/* lower_vec / raise_vec (phys.tools.c:1421, :1487), DOMIXTHETAPHI=0 (metric.h:3) */
void o_lower(const double *ucon, const ogeom *g, double *ucov) {
  ucov[0] = g->gcov[0][0] * ucon[0] + g->gcov[0][1] * ucon[1] + g->gcov[0][2] * ucon[2] + g->gcov[0][3] * ucon[3];
  ucov[1] = g->gcov[0][1] * ucon[0] + g->gcov[1][1] * ucon[1] + g->gcov[1][2] * ucon[2] + g->gcov[1][3] * ucon[3];
  ucov[2] = g->gcov[0][2] * ucon[0] + g->gcov[1][2] * ucon[1] + g->gcov[2][2] * ucon[2];
  ucov[3] = g->gcov[0][3] * ucon[0] + g->gcov[1][3] * ucon[1] + g->gcov[3][3] * ucon[3];
}
void o_raise(const double *ucov, const ogeom *g, double *ucon) {
  ucon[0] = g->gcon[0][0] * ucov[0] + g->gcon[0][1] * ucov[1] + g->gcon[0][2] * ucov[2] + g->gcon[0][3] * ucov[3];
  ucon[1] = g->gcon[0][1] * ucov[0] + g->gcon[1][1] * ucov[1] + g->gcon[1][2] * ucov[2] + g->gcon[1][3] * ucov[3];
  ucon[2] = g->gcon[0][2] * ucov[0] + g->gcon[1][2] * ucov[1] + g->gcon[2][2] * ucov[2] + g->gcon[2][3] * ucov[3];
  ucon[3] = g->gcon[0][3] * ucov[0] + g->gcon[1][3] * ucov[1] + g->gcon[2][3] * ucov[2] + g->gcon[3][3] * ucov[3];
}

/* ---------------------------------------------------------------- state */

/* qsq_calc / gamma_calc_fromuconrel (phys.tools.c:1980, :1955; JONCHECKS off in
   production: qsq clipped at 0) */
double o_qsq(const double *pr, const ogeom *g) {
  double u1 = pr[HARM_U1], u2 = pr[HARM_U2], u3 = pr[HARM_U3];
  return g->gcov[1][1] * u1 * u1 + g->gcov[2][2] * u2 * u2 + g->gcov[3][3] * u3 * u3 +
         2. * (g->gcov[1][2] * u1 * u2 + g->gcov[1][3] * u1 * u3);
}

/* ucon_calc_rel4vel_fromuconrel (phys.tools.c:1900) */
void o_ucon(const double *pr, const ogeom *g, double *ucon, double *gamma, double *qsq) {
  double q = o_qsq(pr, g);
  q = q * (q >= 0.0);
  *qsq = q;
  *gamma = sqrt(1. + q);
  ucon[0] = *gamma / g->alpha;
  for (int j = 1; j < 4; j++) ucon[j] = pr[HARM_U1 + j - 1] - ucon[0] * g->beta[j];
}

/* get_state (phys.tools.c:1513): ucon, ucov, 1+u_t (compute_1plusud0_rel4vel :1272,
   UD0PLUS1FIX=1), b^2 (bsq_calc_fromq_rel4vel :1392), pressure (ideal gas) */
void o_get_state(const double *pr, const ogeom *g, double gam, ostate *q) {
  o_ucon(pr, g, q->ucon, &q->gamma, &q->qsq);
  o_lower(q->ucon, g, q->ucov);
  double ud0tilde = 0.0;
  for (int j = 1; j < 4; j++) ud0tilde += pr[HARM_U1 + j - 1] * g->gcov[0][j];
  double alphasq = g->alpha * g->alpha;
  q->plus1ud0 = ud0tilde + (g->gcovpert_tt - alphasq * (g->betasqoalphasq + q->qsq)) / (1.0 + q->gamma * g->alpha);
  double Bcon[4] = {0.0, pr[HARM_B1], pr[HARM_B2], pr[HARM_B3]}, Bcov[4];
  for (int jj = 0; jj < 4; jj++) {
    Bcov[jj] = 0.0;
    for (int kk = 1; kk < 4; kk++) Bcov[jj] += Bcon[kk] * g->gcov[jj][kk];
  }
  double Bsq = 0.0, udotB = 0.0;
  for (int kk = 1; kk < 4; kk++) Bsq += Bcon[kk] * Bcov[kk];
  for (int kk = 1; kk < 4; kk++) udotB += Bcon[kk] * q->ucov[kk];
  q->bsq = (Bsq + udotB * udotB) / (q->ucon[0] * q->ucon[0]);
  q->pressure = (gam - 1.) * pr[HARM_UU];
}

/* primtoflux (phys.tools.c:30) in UEVOLVE form: mass flux, matter stress with the rest
   mass removed from the energy row (mhd_calc_norestmass_ma :1071), primitive-field EM
   stress (mhd_calc_primfield_em :1133), field flux (dualfullfaraday_calc PRIMMAXWELL
   :392), all times sqrt(-g) (UtoU_gen_allgdet_fromunothing :708). */
void o_primtoflux(const double *pr, const ostate *q, int dir, const ogeom *g, double *F) {
  double ma[4], em[4];
  double rho = pr[HARM_RHO], u = pr[HARM_UU], P = q->pressure, w = P + rho + u;
  ma[0] = (P + u) * q->ucon[dir] * q->ucov[0] + rho * q->ucon[dir] * q->plus1ud0;
  for (int j = 1; j < 4; j++) ma[j] = w * q->ucon[dir] * q->ucov[j];
  ma[dir] += P;
  double Bcon[4] = {0.0, pr[HARM_B1], pr[HARM_B2], pr[HARM_B3]}, Bcov[4];
  for (int jj = 0; jj < 4; jj++) {
    Bcov[jj] = 0.0;
    for (int kk = 1; kk < 4; kk++) Bcov[jj] += Bcon[kk] * g->gcov[jj][kk];
  }
  double Bsq = 0.0, udotB = 0.0;
  for (int kk = 1; kk < 4; kk++) Bsq += Bcon[kk] * Bcov[kk];
  for (int kk = 1; kk < 4; kk++) udotB += Bcon[kk] * q->ucov[kk];
  for (int mu = 0; mu < 4; mu++)
    em[mu] = Bsq * q->ucon[dir] * q->ucov[mu] - Bcon[dir] * Bcov[mu] -
             udotB * (Bcon[dir] * q->ucov[mu] + Bcov[mu] * q->ucon[dir]);
  em[dir] += 0.5 * (Bsq + udotB * udotB);
  double oneovergammasq = 1.0 / (q->ucon[0] * q->ucon[0]);
  for (int mu = 0; mu < 4; mu++) em[mu] *= oneovergammasq;
  double f[HARM_NPR];
  f[HARM_RHO] = rho * q->ucon[dir];
  for (int mu = 0; mu < 4; mu++) f[HARM_UU + mu] = ma[mu] + em[mu];
  if (dir > 0) {
    for (int j = 1; j < 4; j++)
      f[HARM_B1 + j - 1] = (pr[HARM_B1 + j - 1] * q->ucon[dir] - pr[HARM_B1 + dir - 1] * q->ucon[j]) / q->ucon[0];
  } else {
    for (int j = 1; j < 4; j++) f[HARM_B1 + j - 1] = pr[HARM_B1 + j - 1];
  }
  for (int pl = 0; pl < HARM_NPR; pl++) F[pl] = f[pl] * g->gdet;
}

/* vchar (vchar.c:34) with simplefast (vchar.c:260, USESASHAREWRITE=1), TRUEFAST=0 */
int o_vchar(const double *pr, const ostate *q, int dir, const ogeom *g, double gam,
            double *vmax, double *vmin) {
  double rho = pr[HARM_RHO], u = pr[HARM_UU];
  if (u < 0) u = 0;
  if (rho < 0) rho = O_SMALL;
  double P = q->pressure, WW = rho + u + P, cs2;
  if (WW > 0.0) {
    double pp = (gam - 1.) * u, h = rho + u + pp;
    cs2 = gam * pp / h; /* cs2_compute_idealgas (idealgaseos.c:48) */
  } else WW = cs2 = O_SMALL;
  if (cs2 >= 1.0) cs2 = 1.0 - DBL_EPSILON * 10.0;
  else if (cs2 <= 0.0) cs2 = O_SMALL;
  double EF = O_SMALL + fabs(q->bsq + WW);
  double va2 = q->bsq / EF;
  double cms2 = cs2 + va2 - cs2 * va2;
  if (cms2 < 0.0 && cms2 / (cs2 + va2) > -DBL_EPSILON * 100.0) cms2 = 0.0;
  if (cms2 > 1.0 && (cms2 < 1.0 + DBL_EPSILON * 100.0 || rho < 0.0)) cms2 = 1.0;
  /* simplefast: A = e^dir (covariant unit), B = e^t */
  double Asq = g->gcon[dir][dir], Bsq = g->gcon[0][0], AB = g->gcon[dir][0];
  double Au = q->ucon[dir], Bu = q->ucon[0];
  double Au2 = Au * Au, Bu2 = Bu * Bu, AuBu = Au * Bu;
  double B = 2. * (AuBu * (1.0 - cms2) - AB * cms2);
  double A = Bu2 * (1.0 - cms2) - Bsq * cms2;
  double discr = 4.0 * cms2 * ((AB * AB - Asq * Bsq) * cms2 + (2.0 * AB * Au * Bu - Asq * Bu2 - Bsq * Au2) * (cms2 - 1.0));
  if (discr < 0.0) discr = 0.0;
  discr = sqrt(discr);
  double vm = -(-B + discr) / (2. * A), vp = -(-B - discr) / (2. * A);
  if (vp < vm) { *vmax = vm; *vmin = vp; }
  else { *vmax = vp; *vmin = vm; }
  return (!isfinite(vm) || !isfinite(vp));
}

/* source_conn (phys.c:132): dU^{UU+l} += T^j_k Gamma^k_{l j} - rho u^j Gamma^t_{l j},
   times sqrt(-g); mhd_calc uses the rest-mass-removed energy row. */
void o_source(const double *pr, const ostate *q, const ogeom *g, const double *conn, double *dU) {
  double mhd[4][4];
  for (int j = 0; j < 4; j++) {
    double F[HARM_NPR];
    ogeom gn = *g;
    gn.gdet = 1.0;
    o_primtoflux(pr, q, j, &gn, F);
    for (int k = 0; k < 4; k++) mhd[j][k] = F[HARM_UU + k];
  }
  double dUconn[HARM_NPR] = {0};
  for (int l = 0; l < 4; l++)
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 4; k++) dUconn[HARM_UU + l] += mhd[j][k] * conn[(k * 4 + l) * 4 + j];
  for (int l = 0; l < 4; l++)
    for (int j = 0; j < 4; j++) dUconn[HARM_UU + l] += -pr[HARM_RHO] * q->ucon[j] * conn[(0 * 4 + l) * 4 + j];
  for (int pl = 0; pl < HARM_NPR; pl++) dU[pl] = g->gdet * dUconn[pl];
}

void orc_primtoU_point(const double *geomrec, const double *pr, double *U) {
  ogeom g; ostate q;
  og_from_record(geomrec, &g);
  o_get_state(pr, &g, 4.0 / 3.0, &q);
  o_primtoflux(pr, &q, 0, &g, U);
}

void orc_primtoflux_point(const double *geomrec, const double *pr, int dir, double *F) {
  ogeom g; ostate q;
  og_from_record(geomrec, &g);
  o_get_state(pr, &g, 4.0 / 3.0, &q);
  o_primtoflux(pr, &q, dir, &g, F);
}

void orc_vchar_point(const harm_grid *hg, const double *geomrec, const double *pr, int dir,
                     double *vmax, double *vmin) {
  ogeom g; ostate q;
  og_from_record(geomrec, &g);
  o_get_state(pr, &g, hg->gam, &q);
  o_vchar(pr, &q, dir, &g, hg->gam, vmax, vmin);
}

/* ---------------------------------------------------------------- inversion */

#define NUMEPS DBL_EPSILON
#define NEWT_TOL (1E3 * NUMEPS)              /* u2p_defs.h:37 (PRECISEINVERSION) */
#define NEWT_TOL_ULTRAREL (NUMEPS)
#define MIN_NEWT_TOL (1E-6)
#define MAX_NEWT_ITER 200
#define ITERDAMPSTART 10
#define EXTRA_NEWT_ITER 2
#define EXTRA_NEWT_ITER_ULTRAREL 4
#define GAMMASQCHECKRESID (1e2)
#define VERYBIG_D (1.e150)
#define KINDASMALL_D (1.e-100)
#define BIG_D (1.e100)
#define SQRTMINNUMREP (1.4916681462400413e-154) /* sqrt(DBL_MIN) */

enum { EOM_HOT = 0, EOM_COLD = 1 };

typedef struct inv_consts {
  double Bsq, QdotB, QdotBsq, Qtsq, Qdotn, Qdotnp, D;
  double wglobal[3];
  double gam, gammasq_too_big, utsq_too_big;
  int eomtype;
} inv_consts;

/* utsq_calc (utoprim_jon.c:1723) */
static double utsq_calc(double W, const inv_consts *c) {
  double SoW = c->QdotB / W;
  double top = c->Qtsq + (c->Bsq + 2.0 * W) * SoW * SoW;
  double bot = (c->Bsq * c->Bsq - c->Qtsq) + 2.0 * c->Bsq * W + W * W - SoW * SoW * (c->Bsq + 2.0 * W);
  return top / bot;
}
/* vsqgtr1 (utoprim_jon.c:1709) */
static int vsqgtr1(double W, const inv_consts *c) {
  return W * W * W * (W + 2. * c->Bsq) - c->QdotBsq * (2. * W + c->Bsq) <= W * W * (c->Qtsq - c->Bsq * c->Bsq);
}
/* dvsq_dW (utoprim_jon.c:1791) */
static double dvsq_dW(double W, const inv_consts *c) {
  double X = c->Bsq + W, W3 = W * W * W, X3 = X * X * X;
  return -2.0 / X3 * (c->Qtsq + c->QdotBsq * (3.0 * W * X + c->Bsq * c->Bsq) / W3);
}
/* coldgrhd (utoprim_jon.c:1806) */
static int coldgrhd(int8_t *lpflag, double Qtsq, double D, double *Wp) {
  double det = D * D + Qtsq;
  if (det < 0.0) { *lpflag = HARM_UTOPRIMFAILCONVUTSQ; return 1; }
  if (D > 0.0) *Wp = Qtsq / (D + sqrt(det));
  else *Wp = Qtsq / (D - sqrt(det));
  return 0;
}

/* func_Eprime_opt (utoprim_jon.c:2953) with the ideal-gas p(rho0,chi) */
static void func_Eprime(double Wp, const inv_consts *c, double *resid, double *jac, double *dx, double *f) {
  double W = Wp + c->D, X = c->Bsq + W + O_SMALL, X2 = X * X, X3 = X2 * X;
  double utsq = utsq_calc(W, c);
  double gammasq = 1.0 + utsq, gamma = sqrt(gammasq);
  double wmrho0 = (Wp - c->D * utsq / (1.0 + gamma)) / gammasq;
  if (utsq < -0.9 * c->utsq_too_big || utsq != utsq) {
    *resid = -VERYBIG_D; *jac = 0.0; *dx = VERYBIG_D;
    *f = 0.5 * (*resid) * (*resid);
    return;
  }
  double gam = c->gam, igammar = (gam - 1.0) / gam;
  double pofchi = igammar * wmrho0, dpdrho = 0.0, dpdchi = (gam - 1.0) / gam;
  double Ep = c->Qdotnp + Wp - pofchi + 0.5 * c->Bsq + 0.5 * (c->Bsq * c->Qtsq - c->QdotBsq) / X2;
  if (pofchi != pofchi || Ep != Ep) Ep = -VERYBIG_D;
  double dvsq = dvsq_dW(W, c);
  double dwmrho0dW = 1.0 / gammasq, drho0dW = 0.0;
  double dwmrho0dvsq = (c->D * (gamma * 0.5 - 1.0) - Wp), drho0dvsq = -c->D * gamma * 0.5;
  double dpdW = drho0dW * dpdrho + dwmrho0dW * dpdchi;
  double dpdvsq = drho0dvsq * dpdrho + dwmrho0dvsq * dpdchi;
  double dpdWp = dpdW + dpdvsq * dvsq;
  double dE = (1.0 - dpdWp) - (c->Bsq * c->Qtsq - c->QdotBsq) / X3;
  if (dvsq != dvsq || dpdW != dpdW || dpdvsq != dpdvsq || dpdWp != dpdWp || dE != dE) dE = 0.0;
  *resid = Ep; *jac = dE; *dx = -Ep / dE;
  *f = 0.5 * Ep * Ep;
}

/* func_Psq with Psq_Wp / dPsqdWp_Wp (utoprim_jon.c:3108, :1867, :1885) */
static void func_Psq(double Wp, const inv_consts *c, double *resid, double *jac, double *dx, double *f) {
  double W = Wp + c->D, Y = c->Bsq + 2.0 * W, W2 = W * W, S = c->QdotB, D = c->D, Bsq = c->Bsq;
  double r = -c->Qtsq * W2 + Wp * (D + W) * (W2 + Bsq * Y) - Y * S * S;
  double d = 2.0 * (D * ((Bsq + D) * (Bsq + D) - c->Qtsq) - (S * S) + ((Bsq + D) * (Bsq + 5.0 * D) - c->Qtsq) * Wp +
                    3.0 * (Bsq + 2.0 * D) * (Wp * Wp) + 2.0 * (Wp * Wp * Wp));
  *resid = r; *jac = d; *dx = -r / d;
  *f = 0.5 * r * r;
}

static void func_any(double Wp, const inv_consts *c, double *resid, double *jac, double *dx, double *f) {
  if (c->eomtype == EOM_HOT) func_Eprime(Wp, c, resid, jac, dx, f);
  else func_Psq(Wp, c, resid, jac, dx, f);
}

/* validate_Wp (utoprim_jon.c:2319) */
static void validate_Wp(double Wpold, double *Wpnew, const inv_consts *c) {
  if (*Wpnew < -c->D && c->D > 0.0) {
    int8_t vflag = 0;
    double Wp = *Wpnew / 10.0;
    coldgrhd(&vflag, c->Qtsq, c->D, &Wp);
    *Wpnew = Wp * 10.0;
  }
  *Wpnew = (fabs(*Wpnew / c->wglobal[1]) > c->gammasq_too_big) ? 0.5 * (Wpold + *Wpnew) : *Wpnew;
}

/* newt_errorcheck / newt_extracheck (utoprim_jon.c:4488, :4503) */
static int newt_ultrarel(double x0, const inv_consts *c) {
  return (fabs(c->wglobal[1]) > c->wglobal[2]) || (fabs(x0) > c->wglobal[2]);
}
static int newt_errorcheck(double errx, double x0, const inv_consts *c) {
  return newt_ultrarel(x0, c) ? (fabs(errx) <= NEWT_TOL_ULTRAREL) : (fabs(errx) <= NEWT_TOL);
}
static int newt_extracheck(double x0, const inv_consts *c) {
  return newt_ultrarel(x0, c) ? EXTRA_NEWT_ITER_ULTRAREL : EXTRA_NEWT_ITER;
}

/* general_newton_raphson (utoprim_jon.c:3853), n=1, no line search (USE_LINE_SEARCH=-2),
   JONGENNEWTSTUFF=1, NEWCONVERGE=1 */
static int newton(int8_t *lpflag, double *xio, const inv_consts *c, int *lntries, int *nstroke) {
  double x = *xio, x_old = x, x_older = x;
  double dx, dx_old = VERYBIG_D, resid, jac, f = 1.0, errx = 1.0;
  double damp = 1.0;
  int n_iter = 0, keep = 1, diddamp = 0, i_extra = 0, doing_extra = 0;
  while (keep) {
    (*nstroke)++;
    (*lntries)++;
    if (*lntries > ITERDAMPSTART && diddamp == 0) damp = 0.5;
    func_any(x, c, &resid, &jac, &dx, &f);
    x_older = x_old;
    x_old = x;
    diddamp = 0;
    if (n_iter == 0) {
      x_older = x; x_old = x; dx_old = dx;
    } else {
      if (resid <= -VERYBIG_D || jac == 0.0) {
        damp = 0.5 * damp;
        x = x_older;
        dx = dx_old;
        diddamp = 1;
      }
      if (diddamp) {
        func_any(x, c, &resid, &jac, &dx, &f);
        if (resid <= -VERYBIG_D || jac == 0.0) { *xio = x; return 1; }
        x_older = x; x_old = x; dx_old = dx;
      }
    }
    x += damp * dx;
    errx = (c->wglobal[0] == 0.) ? fabs(dx_old) : fabs(dx_old / fmax(fabs(c->wglobal[0]), fabs(x)));
    validate_Wp(x_old, &x, c);
    dx_old = dx;
    if (newt_errorcheck(errx, x, c) && doing_extra == 0 && newt_extracheck(x, c) > 0) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if ((newt_errorcheck(errx, x, c) && doing_extra == 0) || (i_extra > newt_extracheck(x, c)) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(x) || !isfinite(f) || !isfinite(-2.0 * f)) {
    *lpflag = HARM_UTOPRIMFAILNANRESULT;
    *xio = x;
    return 1;
  }
  x = x_old;
  *xio = x;
  if (newt_errorcheck(errx, x, c)) return 0;
  if (fabs(errx) > MIN_NEWT_TOL) { *lpflag = HARM_UTOPRIMFAILCONVRET + 4; return 1; }
  return 0;
}

/* Utoprim_new_body (utoprim_jon.c:406) for the hot (E'(W')) or cold (P^2(W')) equation.
   U and prim here are already alpha-scaled (Utoprim_jon_nonrelcompat_inputnorestmass
   :136).  Returns retval of the reference. */
/* compute_setup_quantities (utoprim_jon.c:716) on alpha-scaled U */
static void setup_quantities(const double *U, const ogeom *g, inv_consts *c, double *Bcon, double *Qtcon) {
  double Bcov[4], ncov[4], ncon[4], Qcovp[4], Qconp[4], Qtcov[4], Qcov[4], Qcon[4];
  c->D = U[HARM_RHO];
  Bcon[0] = 0.;
  for (int i = 1; i < 4; i++) Bcon[i] = U[HARM_B1 + i - 1];
  o_lower(Bcon, g, Bcov);
  c->Bsq = 0.;
  for (int i = 1; i < 4; i++) c->Bsq += Bcon[i] * Bcov[i];
  ncov[0] = -g->alpha; ncov[1] = ncov[2] = ncov[3] = 0.;
  o_raise(ncov, g, ncon);
  for (int i = 0; i < 4; i++) Qcovp[i] = U[HARM_UU + i];
  o_raise(Qcovp, g, Qconp);
  for (int j = 0; j < 4; j++) Qtcon[j] = 0.0;
  for (int j = 1; j < 4; j++)
    for (int i = 1; i < 4; i++) Qtcon[j] += U[HARM_UU + i] * (g->gcon[i][j] + ncon[i] * ncon[j]);
  o_lower(Qtcon, g, Qtcov);
  c->Qtsq = 0.;
  for (int i = 0; i < 4; i++) c->Qtsq += Qtcov[i] * Qtcon[i];
  for (int i = 0; i < 4; i++) Qcov[i] = (i == 0) ? Qcovp[i] - c->D : Qcovp[i];
  o_raise(Qcov, g, Qcon);
  c->QdotB = 0.;
  for (int i = 1; i < 4; i++) c->QdotB += Qcov[i] * Bcon[i];
  c->QdotBsq = c->QdotB * c->QdotB;
  double alpha = g->alpha, alphasq = alpha * alpha;
  double Dfactor = (-g->gcovpert_tt + alphasq * g->betasqoalphasq) / (alphasq + alpha);
  c->Qdotnp = Qconp[0] * ncov[0] + c->D * Dfactor;
  c->Qdotn = Qcon[0] * ncov[0];
}

static int new_body(int eomtype, int8_t *lpflag, const double *U, const ogeom *g, double *prim,
                    double gam, double gammafail, int *lntries, int *nstroke, double *Wp_guess_io,
                    int use_guess) {
  inv_consts c;
  memset(&c, 0, sizeof(c));
  c.eomtype = eomtype;
  c.gam = gam;
  c.gammasq_too_big = gammafail * gammafail;
  c.utsq_too_big = (gammafail - 1.0) * (gammafail - 1.0);
  *lpflag = HARM_UTOPRIMNOFAIL;
  int retval = 0;
  double Bcon[4], Qtcon[4];
  for (int i = HARM_B1; i <= HARM_B3; i++) prim[i] = U[i];
  setup_quantities(U, g, &c, Bcon, Qtcon);

  /* set_guess_Wp (utoprim_jon.c:890) */
  double Wp_last, W_last;
  {
    double utsq = 0.;
    for (int i = 1; i < 4; i++)
      for (int j = 1; j < 4; j++) utsq += g->gcov[i][j] * prim[HARM_U1 + i - 1] * prim[HARM_U1 + j - 1];
    if ((utsq < 0.) && (fabs(utsq) < fabs(-0.9 * c.utsq_too_big))) utsq = 0.0;
    if (!(utsq >= 0. && utsq < c.utsq_too_big)) utsq = 0.0;
    double gammasq = 1. + utsq, gamma = sqrt(gammasq), rho0 = c.D / gamma, u = prim[HARM_UU];
    double p = (gam - 1.) * u;
    double bc[4] = {0.0, prim[HARM_B1], prim[HARM_B2], prim[HARM_B3]}, bcv[4];
    o_lower(bc, g, bcv);
    double bsq = 0.0;
    for (int jj = 1; jj < 4; jj++) bsq += bc[jj] * bcv[jj];
    bsq *= (g->alpha * g->alpha) / gammasq;
    Wp_last = c.D * utsq / (1.0 + gamma) + (u + p) * gammasq;
    double Wpabs = fabs(c.D * utsq) / (1.0 + fabs(gamma)) + (fabs(u) + fabs(p)) * fabs(gammasq) + SQRTMINNUMREP;
    double nuabs = fabs(u) + fabs(p) + fabs(bsq), etaabs = fabs(rho0) + nuabs;
    c.wglobal[2] = GAMMASQCHECKRESID * fabs(rho0);
    if (gammasq * etaabs >= c.wglobal[2]) {
      double Wpcoldhd;
      if (coldgrhd(lpflag, c.Qtsq, c.D, &Wpcoldhd)) Wpcoldhd = Wp_last;
      c.wglobal[0] = fmax(fmax(Wpcoldhd, Wp_last), Wpabs);
      Wp_last = fmax(2.0 * Wpcoldhd, Wp_last);
    } else c.wglobal[0] = Wpabs;
    c.wglobal[1] = fabs(rho0) + c.wglobal[0] + SQRTMINNUMREP;
    if (use_guess) Wp_last = *Wp_guess_io; /* learned guess replaces the previous-state W' */
    W_last = Wp_last + c.D;
    /* verify_Wlast (utoprim_jon.c:1120) */
    if (W_last < -(c.D) || Wp_last < 0) { W_last = -(c.D); Wp_last = 0; }
    for (int inc = 0; vsqgtr1(W_last, &c) && inc < 10; inc++) {
      Wp_last *= 10.;
      W_last = Wp_last + c.D;
    }
    int attempts = 0;
    while (1) {
      double ut2 = utsq_calc(W_last, &c);
      if (ut2 >= 0.0 && ut2 == ut2) break;
      int8_t coldpflag = 0;
      double coldWp = Wp_last;
      coldgrhd(&coldpflag, c.Qtsq, c.D, &coldWp);
      if (Wp_last < coldWp) Wp_last = coldWp;
      if (attempts > 0) Wp_last = fmax(fmax(fabs(Wp_last) * 10.0, NUMEPS * 100.0 * fabs(c.D)), KINDASMALL_D);
      W_last = Wp_last + c.D;
      if (attempts > 1000) { *lpflag = HARM_UTOPRIMFAILCONVGUESSUTSQ; retval += 1; break; }
      attempts++;
    }
  }
  *Wp_guess_io = Wp_last;
  /* root find */
  double Wp = Wp_last;
  retval += newton(lpflag, &Wp, &c, lntries, nstroke);
  if (retval == 0) {
    /* check_Wp (utoprim_jon.c:1188): flags only, return value 0 */
    if (Wp == BIG_D) *lpflag = HARM_UTOPRIMFAILCONVRET + 1;
    else if (Wp <= -(c.D)) *lpflag = HARM_UTOPRIMFAILCONVRET + 1;
    else if (Wp / c.wglobal[1] > c.gammasq_too_big) *lpflag = HARM_UTOPRIMFAILCONVW;
    /* Wp2prim (utoprim_jon.c:1346), PRIMFROMVSQ=0 */
    double pr0[HARM_NPR];
    for (int i = HARM_B1; i <= HARM_B3; i++) prim[i] = U[i];
    memcpy(pr0, prim, sizeof(pr0));
    double W = Wp + c.D;
    double utsq = utsq_calc(W, &c), gammasq = 1.0 + utsq, gamma = sqrt(gammasq);
    double wmrho0 = (Wp - c.D * utsq / (1.0 + gamma)) / gammasq;
    double rho0 = c.D / gamma;
    double p = ((gam - 1.0) / gam) * wmrho0, u = wmrho0 - p;
    if ((rho0 <= 0.) || ((p < 0.) && (eomtype != EOM_COLD))) {
      if ((rho0 <= 0.) && (p >= 0.)) *lpflag = HARM_UTOPRIMFAILRHONEG;
      if ((rho0 > 0.) && (p < 0.)) *lpflag = HARM_UTOPRIMFAILUNEG;
      if ((rho0 <= 0.) && (p < 0.)) *lpflag = HARM_UTOPRIMFAILRHOUNEG;
    }
    prim[HARM_RHO] = rho0;
    prim[HARM_UU] = (eomtype == EOM_COLD) ? 0.0 : u;
    for (int i = 1; i < 4; i++)
      prim[HARM_U1 + i - 1] = gamma / (W + c.Bsq) * (Qtcon[i] + c.QdotB * Bcon[i] / W);
    int nan = 0;
    for (int pl = 0; pl <= HARM_U3; pl++)
      if (!isfinite(prim[pl])) nan = 1;
    if (nan) {
      *lpflag = HARM_UTOPRIMFAILNANRESULT;
      memcpy(prim, pr0, sizeof(pr0));
      return 1;
    }
  }
  return retval;
}

/* Utoprim_jon_nonrelcompat_inputnorestmass (utoprim_jon.c:136) on geometry-free U */
static void utoprim_jon(int eomtype, const double *U, const ogeom *g, int8_t *lpflag, double *prim,
                        double gam, double gammafail, int *nstroke, double *Wpguess, int use_guess) {
  int lntries = 0;
  double U_tmp[HARM_NPR], prim_tmp[HARM_NPR];
  for (int i = HARM_B1; i <= HARM_B3; i++) prim[i] = U[i];
  double alpha = g->alpha;
  for (int i = 0; i < HARM_NPR; i++) U_tmp[i] = alpha * U[i];
  for (int i = 0; i < HARM_NPR; i++) prim_tmp[i] = prim[i];
  for (int i = HARM_B1; i <= HARM_B3; i++) prim_tmp[i] = alpha * prim[i];
  int ret = new_body(eomtype, lpflag, U_tmp, g, prim_tmp, gam, gammafail, &lntries, nstroke, Wpguess, use_guess);
  if (ret == 0) {
    for (int i = 0; i <= HARM_U3; i++) prim[i] = prim_tmp[i];
  } else {
    if (*lpflag == HARM_UTOPRIMNOFAIL || *lpflag < 0) *lpflag = (int8_t)(ret + HARM_UTOPRIMFAILCONVRET + 1);
  }
}

/* Utoprimgen (utoprimgen.c:32) from UEVOLVE U: geometry-free U, hot inversion, then the
   HOT2COLD fallback trycoldinversion (utoprimgen.c:594). */
int o_utoprimgen(const double *U, const ogeom *g, double *pr, int8_t *pflag, double gam,
                 double gammafail, int *nstroke) {
  double Ugf[HARM_NPR], Ugf0[HARM_NPR], pr0[HARM_NPR];
  for (int pl = 0; pl < HARM_NPR; pl++) Ugf[pl] = U[pl] * g->igdet;
  for (int pl = 0; pl < HARM_NPR; pl++) { Ugf0[pl] = Ugf[pl]; pr0[pl] = pr[pl]; }
  *pflag = HARM_UTOPRIMNOFAIL;
  double Wpg = 0.0;
  utoprim_jon(EOM_HOT, Ugf, g, pflag, pr, gam, gammafail, nstroke, &Wpg, 0);
  int8_t hotpflag = *pflag;
  if (hotpflag) {
    double prhot[HARM_NPR], prcold[HARM_NPR];
    int8_t coldpflag = 0;
    for (int pl = 0; pl < HARM_NPR; pl++) { prhot[pl] = pr[pl]; Ugf[pl] = Ugf0[pl]; prcold[pl] = pr0[pl]; }
    double Wpc = 0.0;
    utoprim_jon(EOM_COLD, Ugf, g, &coldpflag, prcold, gam, gammafail, nstroke, &Wpc, 0);
    if (coldpflag <= 0) {
      for (int pl = 0; pl < HARM_NPR; pl++) pr[pl] = prcold[pl];
      pr[HARM_UU] = pr0[HARM_UU];
      *pflag = HARM_UTOPRIMFAILU2AVG1;
    } else {
      for (int pl = 0; pl < HARM_NPR; pl++) pr[pl] = prhot[pl];
    }
  }
  return 0;
}

int orc_utoprimgen_point(const harm_grid *hg, const double *geomrec, const double *U, double *pr,
                         int8_t *pflag, int32_t *iters) {
  ogeom g;
  og_from_record(geomrec, &g);
  int nstroke = 0;
  o_utoprimgen(U, &g, pr, pflag, hg->gam, hg->gammafail, &nstroke);
  if (iters) *iters = nstroke;
  return 0;
}

/* ---------------------------------------------------------------- fixups */

/* limit_gamma (fixup.c:2723), GAMMAERGOLIMIT=0, DO_CONSERVE_D=0.  Returns -1 if changed. */
int o_limit_gamma(double gammamax, double *pr, const ogeom *g) {
  if (gammamax <= 1.0) return 0;
  double gamma, qsq, ucon[4];
  o_ucon(pr, g, ucon, &gamma, &qsq);
  if (gamma > gammamax && gamma != 1.0) {
    double pref = (gammamax * gammamax - 1.) / (gamma * gamma - 1.);
    if (pref < 0.0) return 1;
    double f = sqrt(pref);
    pr[HARM_U1] *= f;
    pr[HARM_U2] *= f;
    pr[HARM_U3] *= f;
    return -1;
  }
  return 0;
}

/* inflow_check_rel4vel (fixup.c:3255) for the outer x1 boundary: zero the radial
   4-velocity where it points inward */
void o_inflow_check_x1up(double *pr, const ogeom *g, double gammamax) {
  double ucon[4], gamma, qsq;
  o_ucon(pr, g, ucon, &gamma, &qsq);
  if (!(ucon[1] < 0.)) return;
  pr[HARM_U1] /= gamma;
  pr[HARM_U2] /= gamma;
  pr[HARM_U3] /= gamma;
  double alpha = 1. / sqrt(-g->gcon[0][0]);
  double betacon = g->gcon[0][1] * alpha * alpha;
  pr[HARM_U1] = betacon / alpha;
  double vsq = 0.;
  for (int j = 1; j < 4; j++)
    for (int k = 1; k < 4; k++) vsq += g->gcov[j][k] * pr[HARM_U1 + j - 1] * pr[HARM_U1 + k - 1];
  if (vsq < 0.0 && vsq > -NUMEPS * 100.0) vsq = 0.0;
  if (vsq >= 1.0) vsq = 1.0 - 1.0 / (gammamax * gammamax);
  gamma = 1. / sqrt(1. - vsq);
  pr[HARM_U1] *= gamma;
  pr[HARM_U2] *= gamma;
  pr[HARM_U3] *= gamma;
}

/* fixup1zone (fixup.c:561), FIXUPTYPE 1: floors rho >= rho_fl, u >= u_fl; the added
   mass and energy enter at zero relative velocity and the cell is re-inverted; then
   limit_gamma.  Returns 1 if a floor acted. */
int o_fixup1zone(double *pr, const ogeom *g, double rhofl, double ufl, double gam,
                 double gammamax, double gammafail, int8_t *pflag, int *nstroke) {
  double prfloor[2] = {rhofl, ufl}, prnew[HARM_NPR];
  int did = 0;
  if (prfloor[0] < O_SMALL) prfloor[0] = O_SMALL;
  if (prfloor[1] < O_SMALL) prfloor[1] = O_SMALL;
  for (int pl = 0; pl < HARM_NPR; pl++) prnew[pl] = pr[pl];
  for (int pl = HARM_RHO; pl <= HARM_UU; pl++)
    if (prfloor[pl] > pr[pl]) { did = 1; prnew[pl] = prfloor[pl]; }
  if (did) {
    ostate q, dq;
    double U[HARM_NPR], dU[HARM_NPR], dpr[HARM_NPR] = {0};
    o_get_state(pr, g, gam, &q);
    ogeom g1 = *g;
    g1.gdet = 1.0; /* primtoU(UNOTHING) */
    o_primtoflux(pr, &q, 0, &g1, U);
    for (int pl = HARM_RHO; pl <= HARM_UU; pl++) dpr[pl] = prnew[pl] - pr[pl];
    o_get_state(dpr, g, gam, &dq);
    o_primtoflux(dpr, &dq, 0, &g1, dU);
    for (int pl = 0; pl < HARM_NPR; pl++) U[pl] += dU[pl];
    /* Utoprimgen(OTHERUTOPRIM, UNOTHING): geometry-free input */
    ogeom g2 = *g;
    g2.igdet = 1.0;
    o_utoprimgen(U, &g2, pr, pflag, gam, gammafail, nstroke);
    if (*pflag > 0)
      for (int pl = 0; pl < HARM_NPR; pl++) pr[pl] = prnew[pl];
  }
  o_limit_gamma(gammamax, pr, g);
  return did;
}

/* the alpha-scaled setup invariants {D, B^2, Qt^2, (Q.B)^2, Q.n'} of geometry-free U */
void o_inv_invariants(const double *Ugf, const ogeom *g, double *out) {
  double U[HARM_NPR], Bcon[4], Qtcon[4];
  inv_consts c;
  memset(&c, 0, sizeof(c));
  for (int i = 0; i < HARM_NPR; i++) U[i] = g->alpha * Ugf[i];
  setup_quantities(U, g, &c, Bcon, Qtcon);
  out[0] = c.D;
  out[1] = c.Bsq;
  out[2] = c.Qtsq;
  out[3] = c.QdotBsq;
  out[4] = c.Qdotnp;
}
