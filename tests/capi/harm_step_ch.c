/* A C caller of libharm_b200 with HARM's own array layout, compiled against
 * include/harm_b200.h alone (tests/test_capi_program.py builds and runs it).
 *
 * It does what HARM's step_ch.c does around the replaced functions: HARM-layout arrays
 * ([k][j][i][pl], ORDERSTORAGE 5) in device memory, converted at the boundary; bound_prim;
 * the initial dt from fluxcalc's three limits; the two RK2 substeps of step_ch_simplempi with
 * advance(), bound_prim, post_fixup(), bound_prim; the state converted back and the flags
 * copied into HARM's int pflag[cell][NUMPFLAGS].  The same step is then taken through the
 * host-buffer entry point over a host array in HARM's layout, and the two results must agree
 * bit for bit.  Exit status 0 on success. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "harm_b200.h"

#define NUMPFLAGS 3

static int fail(const char *what, int rc) {
  fprintf(stderr, "FAIL %s (%d): %s\n", what, rc, harm_b200_last_error());
  return 1;
}

#define MYFUN(call, what)             \
  do {                                \
    int rc_ = (call);                 \
    if (rc_) return fail(what, rc_);  \
  } while (0)

#define CUDA(call)                                                                 \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      fprintf(stderr, "FAIL %s: %s\n", #call, cudaGetErrorString(e_));             \
      return 1;                                                                    \
    }                                                                              \
  } while (0)

int main(void) {
  harm_grid g;
  MYFUN(harm_grid_setup(&g, 32, 24, 16, HARM_LIM_WENO5, 0.9375, 0.3, 40.0, 0.8), "harm_grid_setup");
  const size_t plane = (size_t)g.n1e * g.n2e, cells = plane * g.n3e;
  double *geom = malloc(sizeof(double) * HARM_NLOC * HARM_NGF * plane);
  double *conn = malloc(sizeof(double) * 64 * plane);
  double *aux = malloc(sizeof(double) * HARM_NAUX * plane);
  double *P = calloc(HARM_NPR * cells, sizeof(double));
  double *Pharm = malloc(sizeof(double) * HARM_NPR * cells);
  double *A = malloc(sizeof(double) * HARM_NPR * cells);
  int32_t *hflag = malloc(sizeof(int32_t) * NUMPFLAGS * cells);
  int8_t *flag = malloc(cells);
  if (!geom || !conn || !aux || !P || !Pharm || !A || !hflag || !flag) return 1;
  MYFUN(harm_geometry_build(&g, geom, conn, aux), "harm_geometry_build");
  MYFUN(harm_torus_init(&g, geom, aux, 100.0, 12345, P), "harm_torus_init");
  /* HARM's own p[k][j][i][pl] */
  for (size_t c = 0; c < cells; c++)
    for (int pl = 0; pl < HARM_NPR; pl++) Pharm[c * HARM_NPR + pl] = P[(size_t)pl * cells + c];

  harm_ctx *ctx = NULL;
  MYFUN(harm_b200_create(&g, geom, conn, aux, 0, &ctx), "harm_b200_create");
  double *d_harm, *d_P, *d_pk, *d_F[3];
  int8_t *d_pflag;
  int32_t *d_hflag;
  CUDA(cudaMalloc((void **)&d_harm, sizeof(double) * HARM_NPR * cells));
  CUDA(cudaMalloc((void **)&d_P, sizeof(double) * HARM_NPR * cells));
  CUDA(cudaMalloc((void **)&d_pk, sizeof(double) * HARM_NPR * cells));
  for (int d = 0; d < 3; d++) CUDA(cudaMalloc((void **)&d_F[d], sizeof(double) * HARM_NPR * cells));
  CUDA(cudaMalloc((void **)&d_pflag, cells));
  CUDA(cudaMemset(d_pflag, 0, cells));
  CUDA(cudaMalloc((void **)&d_hflag, sizeof(int32_t) * NUMPFLAGS * cells));
  CUDA(cudaMemset(d_hflag, 0, sizeof(int32_t) * NUMPFLAGS * cells));

  /* HARM's arrays at the boundary; bound_prim */
  CUDA(cudaMemcpy(d_harm, Pharm, sizeof(double) * HARM_NPR * cells, cudaMemcpyHostToDevice));
  MYFUN(harm_b200_from_harm_layout(ctx, d_harm, d_P), "from_harm_layout");
  MYFUN(harm_b200_bound(ctx, d_P), "bound");
  /* the state the host-buffer step starts from: the bounded one, in HARM's layout */
  MYFUN(harm_b200_to_harm_layout(ctx, d_P, d_harm), "to_harm_layout");
  CUDA(cudaDeviceSynchronize());
  CUDA(cudaMemcpy(Pharm, d_harm, sizeof(double) * HARM_NPR * cells, cudaMemcpyDeviceToHost));

  /* initial dt: 1/(1/ndt1 + 1/ndt2 + 1/ndt3) of fluxcalc's limits (prepare_globaldt) */
  double ndt3[3];
  MYFUN(harm_b200_fluxcalc(ctx, HARM_PREC_FP64, d_P, d_F[0], d_F[1], d_F[2], ndt3), "fluxcalc");
  const double dt = 1.0 / (1.0 / ndt3[0] + 1.0 / ndt3[1] + 1.0 / ndt3[2]);

  /* the RK2 midpoint step of setup_rktimestep (step_ch.c:1244-1266) */
  static const double CUf[2][4] = {{1.0, 0.0, 0.5, 0.0}, {1.0, 0.0, 1.0, 0.0}};
  static const double Cun[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 1.0, 0.5}};
  harm_stats st;
  memset(&st, 0, sizeof st);
  double ndt0, ndt1;
  MYFUN(harm_b200_advance(ctx, HARM_PREC_FP64, HARM_GUESS_PREV, 0, 2, d_P, d_P, d_pk, d_pflag, dt, CUf[0], Cun[0],
                          &ndt0, &st), "advance 0");
  MYFUN(harm_b200_bound(ctx, d_pk), "bound");
  MYFUN(harm_b200_post_fixup(ctx, d_pk, d_pflag, 0), "post_fixup 0");
  MYFUN(harm_b200_bound(ctx, d_pk), "bound");
  MYFUN(harm_b200_advance(ctx, HARM_PREC_FP64, HARM_GUESS_PREV, 1, 2, d_P, d_pk, d_P, d_pflag, dt, CUf[1], Cun[1],
                          &ndt1, &st), "advance 1");
  MYFUN(harm_b200_bound(ctx, d_P), "bound");
  MYFUN(harm_b200_post_fixup(ctx, d_P, d_pflag, 1), "post_fixup 1");
  MYFUN(harm_b200_bound(ctx, d_P), "bound");
  MYFUN(harm_b200_to_harm_layout(ctx, d_P, d_harm), "to_harm_layout");
  MYFUN(harm_b200_flags_to_harm(ctx, d_pflag, d_hflag, NUMPFLAGS), "flags_to_harm");
  CUDA(cudaDeviceSynchronize());
  CUDA(cudaMemcpy(A, d_harm, sizeof(double) * HARM_NPR * cells, cudaMemcpyDeviceToHost));
  CUDA(cudaMemcpy(hflag, d_hflag, sizeof(int32_t) * NUMPFLAGS * cells, cudaMemcpyDeviceToHost));
  CUDA(cudaMemcpy(flag, d_pflag, cells, cudaMemcpyDeviceToHost));
  for (size_t c = 0; c < cells; c++)
    if (hflag[c * NUMPFLAGS] != (int32_t)flag[c] || hflag[c * NUMPFLAGS + 1] != 0) {
      fprintf(stderr, "FAIL flags differ at cell %zu\n", c);
      return 1;
    }

  /* the same step through the host-buffer entry point over HARM's layout */
  double dth = dt;
  harm_stats sth;
  memset(&sth, 0, sizeof sth);
  MYFUN(harm_b200_step_host_harm(ctx, HARM_PREC_FP64, HARM_GUESS_PREV, Pharm, &dth, &sth), "step_host_harm");
  if (memcmp(A, Pharm, sizeof(double) * HARM_NPR * cells) != 0) {
    size_t bad = 0;
    for (size_t q = 0; q < HARM_NPR * cells; q++) bad += A[q] != Pharm[q];
    fprintf(stderr, "FAIL the host-buffer step differs from the advance sequence in %zu values\n", bad);
    return 1;
  }
  const double ndt_seq = fmin(ndt0, ndt1), dt_next = fmin(ndt_seq, g.safe * dt);
  if (dth != dt_next) {
    fprintf(stderr, "FAIL next dt %.17g != %.17g\n", dth, dt_next);
    return 1;
  }
  if (sth.newton_iters != st.newton_iters) {
    fprintf(stderr, "FAIL Newton iterations %.0f != %.0f\n", sth.newton_iters, st.newton_iters);
    return 1;
  }
  printf("OK %dx%dx%d step dt=%.6g newton iterations %.0f\n", g.n1, g.n2, g.n3, dt, st.newton_iters);
  MYFUN(harm_b200_destroy(ctx), "destroy");
  cudaFree(d_harm); cudaFree(d_P); cudaFree(d_pk); cudaFree(d_pflag); cudaFree(d_hflag);
  for (int d = 0; d < 3; d++) cudaFree(d_F[d]);
  free(geom); free(conn); free(aux); free(P); free(Pharm); free(A); free(hflag); free(flag);
  return 0;
}
