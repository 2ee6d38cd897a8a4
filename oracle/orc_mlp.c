/*
 * orc_mlp.c -- TEST INFRASTRUCTURE ONLY (CPU oracle; see harm_oracle.h).
 *
 * Double-precision restatement of the learned inversion guess, used to check the device
 * features, the FP32 forward/backward kernels (gradient check) and the BF16 inference.
 * The network has no counterpart in the reference; its inputs are the setup quantities of
 * compute_setup_quantities (utoprim_jon.c:716, restated in orc_phys.c) and its output
 * replaces the starting W' of set_guess_Wp (utoprim_jon.c:890).
 *
 * Features (slog(x) = sign(x) log(1+|x|)), from the alpha-scaled invariants of U/sqrt(-g):
 *   log D, slog(B^2/D), slog(Qt^2/D^2), slog((Q.B)^2/D^3), slog(-Q.n'/D),
 *   slog(Qt^2/((Q.n')^2+D^2)), alpha, log sqrt(-g), beta^2/alpha^2, g_tt+1.
 * Targets: log(W'/D), log(1+utsq), W' = D utsq/(1+gamma) + (u+p) gamma^2 of the primitives.
 * Network: 10 -> 64 -> 64 -> 64 -> 2, SiLU; parameters W1[10][64] b1 W2[64][64] b2
 * W3[64][64] b3 W4[64][2] b4; normalisation fmu[10] fsd[10] tmu[2] tsd[2].
 * Loss: L = 1/(2n) sum (y - (t - tmu)/tsd)^2.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "harm_oracle.h"
#include "orc_internal.h"

#define NIN 10
#define NH 64
#define NOUT 2
#define OFF_W1 0
#define OFF_B1 (OFF_W1 + NIN * NH)
#define OFF_W2 (OFF_B1 + NH)
#define OFF_B2 (OFF_W2 + NH * NH)
#define OFF_W3 (OFF_B2 + NH)
#define OFF_B3 (OFF_W3 + NH * NH)
#define OFF_W4 (OFF_B3 + NH)
#define OFF_B4 (OFF_W4 + NH * NOUT)
#define NPARAMS (OFF_B4 + NOUT)

int orc_mlp_nparams(void) { return NPARAMS; }

/* slog of a ratio formed in FP64 and taken in FP32 (as the device does) */
static float slog(double x) {
  float xf = (float)fmax(fmin(x, 1e38), -1e38);
  return copysignf(log1pf(fabsf(xf)), xf);
}
static float flog(double x) { return logf(fmaxf((float)fmin(x, 1e38), 1e-38f)); }

void orc_mlp_features(const harm_grid *hg, const double *geomrec, const double *U, const double *P,
                      float *feat, float *targ) {
  ogeom g;
  og_from_record(geomrec, &g);
  double Ugf[HARM_NPR], q[5];
  for (int p = 0; p < HARM_NPR; p++) Ugf[p] = U[p] * g.igdet;
  o_inv_invariants(Ugf, &g, q);
  const double D = (q[0] > 1e-300) ? q[0] : 1e-300, iD = 1.0 / D;
  feat[0] = flog(D);
  feat[1] = slog(q[1] * iD);
  feat[2] = slog(q[2] * iD * iD);
  feat[3] = slog(q[3] * iD * iD * iD);
  feat[4] = slog(-q[4] * iD);
  feat[5] = slog(q[2] / (q[4] * q[4] + D * D));
  feat[6] = (float)g.alpha;
  feat[7] = flog(fabs(g.gdet));
  feat[8] = (float)g.betasqoalphasq;
  feat[9] = (float)g.gcovpert_tt;
  if (targ && P) {
    double utsq = o_qsq(P, &g);
    if (utsq < 0.0) utsq = 0.0;
    const double gamma = sqrt(1.0 + utsq), u = P[HARM_UU], p = (hg->gam - 1.0) * u;
    const double wp = q[0] * utsq / (1.0 + gamma) + (u + p) * (1.0 + utsq);
    const double r = wp / D;
    targ[0] = (float)log(r > 1e-300 ? r : 1e-300);
    targ[1] = (float)log1p(utsq);
  }
}

static double silu(double z) { return z / (1.0 + exp(-z)); }
static double dsilu(double z) {
  double s = 1.0 / (1.0 + exp(-z));
  return s * (1.0 + z * (1.0 - s));
}

/* forward of one sample: z1..z3 pre-activations, y standardised outputs */
static void forward(const double *x, const float *w, double *z1, double *z2, double *z3, double *y) {
  for (int o = 0; o < NH; o++) {
    double z = w[OFF_B1 + o];
    for (int i = 0; i < NIN; i++) z += x[i] * w[OFF_W1 + i * NH + o];
    z1[o] = z;
  }
  for (int o = 0; o < NH; o++) {
    double z = w[OFF_B2 + o];
    for (int k = 0; k < NH; k++) z += silu(z1[k]) * w[OFF_W2 + k * NH + o];
    z2[o] = z;
  }
  for (int o = 0; o < NH; o++) {
    double z = w[OFF_B3 + o];
    for (int k = 0; k < NH; k++) z += silu(z2[k]) * w[OFF_W3 + k * NH + o];
    z3[o] = z;
  }
  for (int o = 0; o < NOUT; o++) {
    double z = w[OFF_B4 + o];
    for (int k = 0; k < NH; k++) z += silu(z3[k]) * w[OFF_W4 + k * NOUT + o];
    y[o] = z;
  }
}

double orc_mlp_loss_grad(int n, const float *feat, const float *targ, const float *params,
                         const float *norm, double *pred, double *grad) {
  if (grad) memset(grad, 0, sizeof(double) * NPARAMS);
  double loss = 0.0;
  for (int s = 0; s < n; s++) {
    double x[NIN], z1[NH], z2[NH], z3[NH], y[NOUT], dy[NOUT];
    for (int i = 0; i < NIN; i++) x[i] = ((double)feat[s * NIN + i] - norm[i]) / norm[NIN + i];
    forward(x, params, z1, z2, z3, y);
    for (int o = 0; o < NOUT; o++) {
      if (pred) pred[s * NOUT + o] = y[o] * norm[2 * NIN + NOUT + o] + norm[2 * NIN + o];
      if (targ) {
        double t = ((double)targ[s * NOUT + o] - norm[2 * NIN + o]) / norm[2 * NIN + NOUT + o];
        double r = y[o] - t;
        loss += 0.5 * r * r / n;
        dy[o] = r / n;
      } else {
        dy[o] = 0.0;
      }
    }
    if (!grad || !targ) continue;
    double d3[NH], d2[NH], d1[NH];
    for (int o = 0; o < NOUT; o++) grad[OFF_B4 + o] += dy[o];
    for (int k = 0; k < NH; k++) {
      double h = silu(z3[k]);
      double dh = 0.0;
      for (int o = 0; o < NOUT; o++) {
        grad[OFF_W4 + k * NOUT + o] += h * dy[o];
        dh += dy[o] * params[OFF_W4 + k * NOUT + o];
      }
      d3[k] = dh * dsilu(z3[k]);
    }
    for (int o = 0; o < NH; o++) grad[OFF_B3 + o] += d3[o];
    for (int k = 0; k < NH; k++) {
      double h = silu(z2[k]), dh = 0.0;
      for (int o = 0; o < NH; o++) {
        grad[OFF_W3 + k * NH + o] += h * d3[o];
        dh += d3[o] * params[OFF_W3 + k * NH + o];
      }
      d2[k] = dh * dsilu(z2[k]);
    }
    for (int o = 0; o < NH; o++) grad[OFF_B2 + o] += d2[o];
    for (int k = 0; k < NH; k++) {
      double h = silu(z1[k]), dh = 0.0;
      for (int o = 0; o < NH; o++) {
        grad[OFF_W2 + k * NH + o] += h * d2[o];
        dh += d2[o] * params[OFF_W2 + k * NH + o];
      }
      d1[k] = dh * dsilu(z1[k]);
    }
    for (int o = 0; o < NH; o++) grad[OFF_B1 + o] += d1[o];
    for (int i = 0; i < NIN; i++)
      for (int o = 0; o < NH; o++) grad[OFF_W1 + i * NH + o] += x[i] * d1[o];
  }
  return loss;
}
