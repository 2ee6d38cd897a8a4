// harm_capi.cu -- the C ABI of libharm_b200.so (include/harm_b200.h): context, uploads,
// and the reference-shaped entry points, each a sequence of launches on the context stream.
//
// Substep order (advance_standard advance.c:140 + post_advance step_ch.c:288):
//   fluxes(p_b) -> EMFs -> update+inversion(p_i, p_b -> p_f) -> bound(p_f) ->
//   bound(pflag) + fixup_utoprim(p_f) -> bound(p_f)
// Full step: two substeps (RK2 midpoint), then dt on the device (prepare_globaldt
// advance.c:1558, post_stepch step_ch.c:213).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include "harm_common.cuh"
#include "harm_paths.h"

static __thread char g_errbuf[512];

int hb_seterr(const char* what, cudaError_t e) {
  snprintf(g_errbuf, sizeof(g_errbuf), "%s: %s", what, cudaGetErrorString(e));
  return 1;
}

static int seterr_msg(const char* msg, int code) {
  snprintf(g_errbuf, sizeof(g_errbuf), "%s", msg);
  return code;
}

int hb_setmsg(const char* msg, int code) { return seterr_msg(msg, code); }

extern "C" const char* harm_b200_last_error(void) { return g_errbuf; }

// the context of grid g on `device` with every buffer allocated; the tables are filled by
// the caller (upload or device build)
static int create_ctx(const harm_grid* g, int device, harm_ctx** out) {
  if (g->lim != HARM_LIM_MC && g->lim != HARM_LIM_PARA && g->lim != HARM_LIM_WENO5 && g->lim != HARM_LIM_PARALINE)
    return seterr_msg("unknown reconstruction", 2);
  if (g->lim == HARM_LIM_WENO5 && g->ng < 6) return seterr_msg("WENO5 needs ng >= 6", 2);
  if (g->lim == HARM_LIM_PARALINE && g->ng < 4) return seterr_msg("PARALINE needs ng >= 4", 2);
  if (g->fluxmethod != HARM_FLUX_HLL && g->fluxmethod != HARM_FLUX_LAXF) return seterr_msg("unknown fluxmethod", 2);
  double mlp_gate = 0.02;  // the gated learned start's threshold (HARM_B200_MLP_GATE)
  if (const char* e = getenv("HARM_B200_MLP_GATE")) {
    char* end = nullptr;
    const double v = strtod(e, &end);
    if (end == e || !(v >= 0.0)) return seterr_msg("HARM_B200_MLP_GATE is not a non-negative number", 2);
    mlp_gate = v;
  }
  harm_ctx* c = new harm_ctx();
  memset((void*)c, 0, sizeof(*c));
  c->g = *g;
  c->device = device;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  Dims d = dims_of(*g);
  c->plane = d.plane;
  c->cells = d.cells;
  size_t gsz = (size_t)HARM_NLOC * HARM_NGF * d.plane;
  CK(cudaMalloc(&c->d_geom, gsz * sizeof(double)));
  CK(cudaMalloc(&c->d_geomf, gsz * sizeof(float)));
  CK(cudaMalloc(&c->d_conn, 64 * d.plane * sizeof(double)));
  CK(cudaMalloc(&c->d_aux, HARM_NAUX * d.plane * sizeof(double)));
  for (int q = 0; q < 3; q++) {
    CK(cudaMalloc(&c->d_F[q], NPR * d.cells * sizeof(double)));
    CK(cudaMalloc(&c->d_Ff[q], NPR * d.cells * sizeof(float)));
  }
  CK(cudaMalloc(&c->d_emf, 3 * d.cells * sizeof(double)));
  CK(cudaMalloc(&c->d_emff, 3 * d.cells * sizeof(float)));
  if (g->lim == HARM_LIM_WENO5) CK(cudaMalloc(&c->d_line, 9 * d.cells * sizeof(double)));
  CK(cudaMalloc(&c->d_pk, NPR * d.cells * sizeof(double)));
  CK(cudaMalloc(&c->d_U, NPR * d.cells * sizeof(double)));
  CK(cudaMalloc(&c->d_rare, (size_t)d.n1 * d.n2 * d.n3 * sizeof(unsigned int)));
  CK(cudaMalloc(&c->d_pflag, d.cells));
  CK(cudaMemset(c->d_pflag, 0, d.cells));
  c->fix_cap = (unsigned int)std::min<size_t>((size_t)d.n1 * d.n2 * d.n3, 0xFFFFFFF0u);
  CK(cudaMalloc(&c->d_fixrec, (size_t)c->fix_cap * sizeof(FixRec)));
  CK(cudaMalloc(&c->d_scal, 64 * sizeof(double)));
  CK(cudaMemset(c->d_scal, 0, 64 * sizeof(double)));
  c->d_dtslots = (unsigned long long*)(c->d_scal + 0);  // 6 slots
  c->d_dt = c->d_scal + 8;
  c->d_ndt = c->d_scal + 9;                             // 2
  c->d_stats = c->d_scal + 16;                          // 5
  c->d_nrec = (unsigned int*)(c->d_scal + 24);
  c->d_nrare = (unsigned int*)(c->d_scal + 25);
  c->d_nhard = (unsigned int*)(c->d_scal + 26);
  c->d_status = (unsigned int*)(c->d_scal + 28);
  {
    // FP32 flux tiles: plain coalesced loads (default) or TMA ("tma"); both feed the same
    // arithmetic.  The TMA-staged kernel measured slower on B200 (it needs ~120 registers for
    // its tile loop, halving the warps that hide the face physics' latency), so it is opt-in.
    const char* e = getenv("HARM_B200_FLUX_STAGING");
    c->flux_tma = (e && strcmp(e, "tma") == 0);
    // learned start: by default ("gated") only for the cells whose previous state is a poor
    // start, the mma.sync network inside the inversion kernel of those cells; for every
    // cell: the mma.sync network as a kernel ahead of the inversion ("mma") or inside the
    // inversion kernel ("mma-fused"), the tcgen05 network as a kernel ahead of it ("tc") or
    // inside the inversion kernel ("tc-fused").  The network's arithmetic is the same in all.
    const char* m = getenv("HARM_B200_MLP_ENGINE");
    c->mlp_tc = (m && strcmp(m, "tc") == 0) ? 1 : (m && strcmp(m, "tc-fused") == 0) ? 2
              : (m && strcmp(m, "mma-fused") == 0) ? 3 : (m && strcmp(m, "mma") == 0) ? 0 : 4;
    c->mlp_gate = mlp_gate;
    CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
  }
  CK(cudaMemset(c->d_dtslots, 0xFF, 6 * sizeof(unsigned long long)));
  CK(cudaMallocHost(&c->h_scal, 64 * sizeof(double)));
  *out = c;
  return 0;
}

extern "C" int harm_b200_create(const harm_grid* g, const double* geom_h, const double* conn_h, const double* aux_h,
                                int device, harm_ctx** out) {
  if (!g || !geom_h || !conn_h || !aux_h || !out) return seterr_msg("null argument", 1);
  harm_ctx* c = nullptr;
  if (int rc = create_ctx(g, device, &c)) return rc;
  const size_t gsz = (size_t)HARM_NLOC * HARM_NGF * c->plane;
  CK(cudaMemcpy(c->d_geom, geom_h, gsz * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_conn, conn_h, 64 * c->plane * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_aux, aux_h, HARM_NAUX * c->plane * sizeof(double), cudaMemcpyHostToDevice));
  if (int rc = hp_geometry_f32(c)) return rc;
  *out = c;
  return 0;
}

extern "C" int harm_b200_create_grid(const harm_grid* g, int device, harm_ctx** out) {
  if (!g || !out) return seterr_msg("null argument", 1);
  harm_ctx* c = nullptr;
  if (int rc = create_ctx(g, device, &c)) return rc;
  if (int rc = hp_geometry_build(c)) return rc;
  if (int rc = hp_geometry_f32(c)) return rc;
  *out = c;
  return 0;
}

extern "C" int harm_b200_get_tables(harm_ctx* c, double* geom_h, double* conn_h, double* aux_h) {
  if (!c) return seterr_msg("null argument", 1);
  const size_t gsz = (size_t)HARM_NLOC * HARM_NGF * c->plane;
  if (geom_h) CK(cudaMemcpy(geom_h, c->d_geom, gsz * sizeof(double), cudaMemcpyDeviceToHost));
  if (conn_h) CK(cudaMemcpy(conn_h, c->d_conn, 64 * c->plane * sizeof(double), cudaMemcpyDeviceToHost));
  if (aux_h) CK(cudaMemcpy(aux_h, c->d_aux, HARM_NAUX * c->plane * sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int harm_b200_destroy(harm_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  void* ptrs[] = {c->d_geom, c->d_geomf, c->d_conn, c->d_aux, c->d_F[0], c->d_F[1], c->d_F[2], c->d_Ff[0], c->d_Ff[1],
                  c->d_Ff[2], c->d_emf, c->d_emff, c->d_line, c->d_Paos, c->d_pk, c->d_U, c->d_rare, c->d_pflag, c->d_fixrec, c->d_scal, c->d_Pdev, c->d_mlp, c->d_wpg,
                  c->d_mlp_master, c->d_mlp_adam, c->d_mlp_work};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->h_scal) cudaFreeHost(c->h_scal);
  if (c->copy_stream) {
    cudaStreamSynchronize(c->copy_stream);
    cudaStreamDestroy(c->copy_stream);
    cudaEventDestroy(c->entry_ev);
    for (int s = 0; s < HARM_H2D_SLABS; s++) cudaEventDestroy(c->slab_ev[s]);
  }
  if (c->d2h_stream) {
    cudaStreamSynchronize(c->d2h_stream);
    cudaStreamDestroy(c->d2h_stream);
    cudaEventDestroy(c->done_ev);
    for (int s = 0; s < HARM_H2D_SLABS; s++) cudaEventDestroy(c->d2h_ev[s]);
  }
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

extern "C" void* harm_b200_stream(harm_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" unsigned long long harm_b200_launch_count(harm_ctx* c) { return c ? c->launches : 0ull; }

extern "C" int harm_b200_bound(harm_ctx* c, double* d_P) { return hp_bound(c, d_P, nullptr); }

extern "C" int harm_b200_fluxcalc(harm_ctx* c, int precision, const double* d_pb, double* d_F1, double* d_F2,
                                  double* d_F3, double ndt[3]) {
  if (precision != HARM_PREC_FP64 && precision != HARM_PREC_FP64_FMA)
    return seterr_msg("fluxcalc into FP64 arrays needs HARM_PREC_FP64 or HARM_PREC_FP64_FMA", 2);
  unsigned long long* slots = c->d_dtslots;
  CK(cudaMemsetAsync(slots, 0xFF, 3 * sizeof(unsigned long long), c->stream));
  if (precision == HARM_PREC_FP64_FMA) {
    if (hp_fluxes_fp64fma(c, d_pb, d_F1, d_F2, d_F3, c->d_emf, slots)) return 1;
  } else if (hp_fluxes_fp64(c, d_pb, d_F1, d_F2, d_F3, c->d_emf, slots)) {
    return 1;
  }
  if (hp_emf_to_flux_fp64(c, c->d_emf, d_F1, d_F2, d_F3)) return 1;
  unsigned long long hb[3];
  CK(cudaMemcpyAsync(hb, slots, sizeof(hb), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int q = 0; q < 3; q++) {
    double v;
    memcpy(&v, &hb[q], 8);
    ndt[q] = (hb[q] == 0xFFFFFFFFFFFFFFFFull) ? 1.e100 : v;
  }
  CK(cudaMemsetAsync(slots, 0xFF, 3 * sizeof(unsigned long long), c->stream));
  return 0;
}

// the learned guess needs a network set by harm_b200_mlp_set
static int check_guess(harm_ctx* c, int guess) {
  if (guess != HARM_GUESS_PREV && guess != HARM_GUESS_MLP) return seterr_msg("unknown guess", 2);
  if (guess == HARM_GUESS_MLP && (!c->d_mlp || !c->mlp_step))
    return seterr_msg("HARM_GUESS_MLP without a network (harm_b200_mlp_set)", 3);
  return 0;
}

// one substep on the device; dt from d_dt, dt minima of this substep into slots
static int check_precision(int precision) {
  if (precision != HARM_PREC_FP64 && precision != HARM_PREC_MIXED && precision != HARM_PREC_FP64_FMA)
    return seterr_msg("unknown precision", 2);
  return 0;
}

// u: the caller's conserved arrays of the RK step (ui, uf, ucum) or NULL
static int substep(harm_ctx* c, int precision, int guess, int timeorder, int numtimeorders, const double* d_pi,
                   const double* d_pb, double* d_pf, int8_t* d_pflag, const double* CUf, const double* Cunew,
                   unsigned long long* slots, bool with_stats, const SlabWait* sw = nullptr,
                   double* const* u = nullptr) {
  if (int rc = check_guess(c, guess)) return rc;
  if (int rc = check_precision(precision)) return rc;
  StepCoef sc{};
  sc.CUf0 = CUf[0]; sc.CUf1 = CUf[1]; sc.CUf2 = CUf[2];
  sc.Cun0 = Cunew[0]; sc.Cun1 = Cunew[1]; sc.Cun2 = Cunew[2];
  sc.finalstep = (timeorder == numtimeorders - 1);
  sc.guess = guess;
  sc.first = (timeorder == 0);
  if (u) { sc.ui = u[0]; sc.uf = u[1]; sc.ucum = u[2]; }
  double* st = with_stats ? c->d_stats : nullptr;
  if (precision == HARM_PREC_FP64) {
    if (hp_fluxes_fp64(c, d_pb, c->d_F[0], c->d_F[1], c->d_F[2], c->d_emf, slots, sw)) return 1;
    return hp_update_fp64(c, sc, d_pi, d_pb, d_pf, d_pflag, st);
  }
  if (precision == HARM_PREC_FP64_FMA) {
    if (hp_fluxes_fp64fma(c, d_pb, c->d_F[0], c->d_F[1], c->d_F[2], c->d_emf, slots, sw)) return 1;
    return hp_update_fp64fma(c, sc, d_pi, d_pb, d_pf, d_pflag, st);
  }
  if (hp_fluxes_mixed(c, d_pb, c->d_Ff[0], c->d_Ff[1], c->d_Ff[2], c->d_emff, slots, sw)) return 1;
  return hp_update_mixed(c, sc, d_pi, d_pb, d_pf, d_pflag, st);
}

// the device error word, read after a synchronisation (it is cleared when reported)
static int check_status(harm_ctx* c) {
  unsigned int st = 0;
  CK(cudaMemcpy(&st, c->d_status, sizeof(st), cudaMemcpyDeviceToHost));
  if (st) {
    CK(cudaMemset(c->d_status, 0, sizeof(st)));
    if (st & 1u) return seterr_msg("a flux tile's TMA load did not complete (the step's fluxes are incomplete)", 5);
    return seterr_msg("a tensor-core MMA of the learned start did not complete (the step's inversion is incomplete)", 5);
  }
  return 0;
}

static void add_stats(harm_ctx* c, harm_stats* stats, double inverted, int guess) {
  if (!stats) return;
  stats->newton_iters += c->h_scal[8];
  stats->cells_inverted += inverted;
  // the gated engine counts the cells it gives the learned start; the others give it to all
  if (guess == HARM_GUESS_MLP) stats->mlp_cells += (c->mlp_tc == 4) ? c->h_scal[9] : inverted;
  stats->mlp_fallbacks += c->h_scal[10];
  stats->inversion_failures += c->h_scal[11];
  stats->floor_hits += c->h_scal[12];
}

extern "C" int harm_b200_advance(harm_ctx* c, int precision, int guess, int timeorder, int numtimeorders,
                                 const double* d_pi, const double* d_pb, double* d_pf, int8_t* d_pflag, double dt,
                                 const double CUf[4], const double Cunew[4], double* ndt, harm_stats* stats) {
  // The conserved state of a substep is formed from U_i and dU alone: U_f = CUf0 U_i +
  // CUf2 dt dU (UFSET global.stepch.h:1 without the CUf1 U_f term) and, on the final
  // substep, ucum = Cunew0 U_i + Cunew1 dt dU + Cunew2 U_f (UCUMUPDATE :10 into an empty
  // ucum).  That is exact for setup_rktimestep's TIMEORDER 1 and its RK2 midpoint; sets that
  // carry U_f or ucum across substeps (TVD RK2, RK3, RK4) are refused here and run through
  // harm_b200_advance_u, which takes the conserved arrays.
  if (timeorder < 0 || numtimeorders < 1 || timeorder >= numtimeorders)
    return seterr_msg("timeorder must lie in [0, numtimeorders)", 2);
  if (CUf[1] != 0.0 || (timeorder < numtimeorders - 1 && (Cunew[0] != 0.0 || Cunew[1] != 0.0 || Cunew[2] != 0.0)))
    return seterr_msg("RK coefficients that carry U_f or ucum across substeps are not supported (CUf[1] must be 0 "
                      "and Cunew[0..2] 0 before the final substep)", 2);
  Dims d = dims_of(c->g);
  c->h_scal[0] = dt;
  CK(cudaMemcpyAsync(c->d_dt, c->h_scal, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->d_stats, 0, 5 * sizeof(double), c->stream));
  if (substep(c, precision, guess, timeorder, numtimeorders, d_pi, d_pb, d_pf, d_pflag, CUf, Cunew, c->d_dtslots, true))
    return 1;
  if (hp_copy_ghosts(c, d_pb, d_pf)) return 1;
  if (hp_finalize_dt(c, nullptr, c->d_ndt, 1)) return 1;
  CK(cudaMemcpyAsync(c->h_scal + 1, c->d_ndt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->h_scal + 8, c->d_stats, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (int rc = check_status(c)) return rc;
  if (ndt) *ndt = c->h_scal[1];
  add_stats(c, stats, (double)d.n1 * d.n2 * d.n3, guess);
  return 0;
}

// advance() with the RK step's conserved arrays (advance.c:85-91): every setup_rktimestep
// coefficient set, U_f and ucum carried across the substeps in the caller's d_uf, d_ucum
extern "C" int harm_b200_advance_u(harm_ctx* c, int precision, int guess, int timeorder, int numtimeorders,
                                   const double* d_pi, const double* d_pb, double* d_pf, int8_t* d_pflag,
                                   double* d_ui, double* d_uf, double* d_ucum, double dt, const double CUf[4],
                                   const double Cunew[4], double* ndt, harm_stats* stats) {
  if (timeorder < 0 || numtimeorders < 1 || timeorder >= numtimeorders)
    return seterr_msg("timeorder must lie in [0, numtimeorders)", 2);
  if (!d_ui || !d_uf || !d_ucum) return seterr_msg("null conserved array", 1);
  Dims d = dims_of(c->g);
  c->h_scal[0] = dt;
  CK(cudaMemcpyAsync(c->d_dt, c->h_scal, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->d_stats, 0, 5 * sizeof(double), c->stream));
  double* const u[3] = {d_ui, d_uf, d_ucum};
  if (substep(c, precision, guess, timeorder, numtimeorders, d_pi, d_pb, d_pf, d_pflag, CUf, Cunew, c->d_dtslots, true,
              nullptr, u))
    return 1;
  if (hp_copy_ghosts(c, d_pb, d_pf)) return 1;
  if (hp_finalize_dt(c, nullptr, c->d_ndt, 1)) return 1;
  CK(cudaMemcpyAsync(c->h_scal + 1, c->d_ndt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->h_scal + 8, c->d_stats, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (int rc = check_status(c)) return rc;
  if (ndt) *ndt = c->h_scal[1];
  add_stats(c, stats, (double)d.n1 * d.n2 * d.n3, guess);
  return 0;
}

extern "C" int harm_b200_post_fixup(harm_ctx* c, double* d_pf, int8_t* d_pflag, int finalstep) {
  return hp_fixup(c, d_pf, d_pflag, finalstep ? 1 : 0);
}

// enqueue one full RK2 step with dt in d_dt (no host synchronisation)
// sw: d_P is still arriving in k-slabs (the first substep's flux launches wait for them)
static int enqueue_step(harm_ctx* c, int precision, int guess, double* d_P, bool with_stats,
                        const SlabWait* sw = nullptr) {
  static const double CUf[2][4] = {{1.0, 0.0, 0.5, 0.0}, {1.0, 0.0, 1.0, 0.0}};
  static const double Cun[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 1.0, 0.5}};
  if (substep(c, precision, guess, 0, 2, d_P, d_P, c->d_pk, c->d_pflag, CUf[0], Cun[0], c->d_dtslots, with_stats, sw))
    return 1;
  // bound_prim of p_f and of the flags in one pass (neither depends on the other), post_fixup,
  // bound_prim (post_advance step_ch.c:288-330)
  if (hp_bound(c, c->d_pk, c->d_pflag)) return 1;
  if (hp_fixup(c, c->d_pk, c->d_pflag, 0, false)) return 1;
  if (hp_bound(c, c->d_pk, nullptr)) return 1;
  if (substep(c, precision, guess, 1, 2, d_P, c->d_pk, d_P, c->d_pflag, CUf[1], Cun[1], c->d_dtslots + 3, with_stats))
    return 1;
  if (hp_bound(c, d_P, c->d_pflag)) return 1;
  if (hp_fixup(c, d_P, c->d_pflag, 1, false)) return 1;
  if (hp_bound(c, d_P, nullptr)) return 1;
  return hp_finalize_dt(c, c->d_dt, c->d_ndt, 2);
}

extern "C" int harm_b200_step_n(harm_ctx* c, int precision, int guess, double* d_P, int nsteps, double* dt,
                                harm_stats* stats) {
  Dims d = dims_of(c->g);
  c->h_scal[0] = *dt;
  CK(cudaMemcpyAsync(c->d_dt, c->h_scal, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (stats) CK(cudaMemsetAsync(c->d_stats, 0, 5 * sizeof(double), c->stream));
  for (int s = 0; s < nsteps; s++)
    if (enqueue_step(c, precision, guess, d_P, stats != nullptr)) return 1;
  CK(cudaMemcpyAsync(c->h_scal, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (stats) CK(cudaMemcpyAsync(c->h_scal + 8, c->d_stats, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (int rc = check_status(c)) return rc;
  *dt = c->h_scal[0];
  add_stats(c, stats, 2.0 * nsteps * (double)d.n1 * d.n2 * d.n3, guess);
  return 0;
}

extern "C" int harm_b200_step(harm_ctx* c, int precision, int guess, double* d_P, double* dt, harm_stats* stats) {
  return harm_b200_step_n(c, precision, guess, d_P, 1, dt, stats);
}

// H2D of the state in at most HARM_H2D_SLABS slabs of k-planes (one cudaMemcpyAsync per
// primitive and slab, each slab followed by an event) on the copy stream, after the context
// stream's earlier work
// harm_layout: h_P is in HARM's [k][j][i][pl] layout (one copy per slab into d_Paos, converted
// into d_Pdev on the context stream after the slab's event)
// after_slab (optional): per slab, an event the slab's copy waits for (the previous step's
// D2H of the same slab, which wrote the host values this copy reads)
static int h2d_slabs(harm_ctx* c, const double* h_P, SlabWait* sw, bool harm_layout = false,
                     const cudaEvent_t* after_slab = nullptr) {
  if (!c->copy_stream) {
    CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->entry_ev, cudaEventDisableTiming));
    for (int s = 0; s < HARM_H2D_SLABS; s++) CK(cudaEventCreateWithFlags(&c->slab_ev[s], cudaEventDisableTiming));
  }
  const int n3e = c->g.n3e;
  const int planes = (n3e + HARM_H2D_SLABS - 1) / HARM_H2D_SLABS;
  const int nslab = (n3e + planes - 1) / planes;
  CK(cudaEventRecord(c->entry_ev, c->stream));
  CK(cudaStreamWaitEvent(c->copy_stream, c->entry_ev, 0));
  for (int s = 0; s < nslab; s++) {
    const int z0 = s * planes, z1 = (z0 + planes < n3e) ? z0 + planes : n3e;
    const size_t off = (size_t)z0 * c->plane, bytes = (size_t)(z1 - z0) * c->plane * sizeof(double);
    if (after_slab) CK(cudaStreamWaitEvent(c->copy_stream, after_slab[s], 0));
    if (harm_layout) {
      CK(cudaMemcpyAsync(c->d_Paos + NPR * off, h_P + NPR * off, NPR * bytes, cudaMemcpyHostToDevice, c->copy_stream));
    } else {
      for (int p = 0; p < NPR; p++)
        CK(cudaMemcpyAsync(c->d_Pdev + (size_t)p * c->cells + off, h_P + (size_t)p * c->cells + off, bytes,
                           cudaMemcpyHostToDevice, c->copy_stream));
    }
    CK(cudaEventRecord(c->slab_ev[s], c->copy_stream));
  }
  sw->ev = c->slab_ev;
  sw->nslab = nslab;
  sw->planes = planes;
  sw->ctx = c;
  sw->aos = harm_layout ? c->d_Paos : nullptr;
  sw->soa = c->d_Pdev;
  return 0;
}

// One full step over a host array: the state goes to the device in k-slabs while the first
// substep's flux tiles of the slabs already resident run, then the rest of the step, then the
// state comes back.  Results are those of harm_b200_step on the same state.  harm_layout: the
// host array is in HARM's [k][j][i][pl] layout (converted on the device as each slab arrives,
// and back before the copy out).
static int step_host(harm_ctx* c, int precision, int guess, double* h_P, double* dt, harm_stats* stats,
                     bool harm_layout) {
  if (int rc = check_guess(c, guess)) return rc;
  if (int rc = check_precision(precision)) return rc;
  Dims d = dims_of(c->g);
  const size_t bytes = NPR * c->cells * sizeof(double);
  if (!c->d_Pdev) CK(cudaMalloc(&c->d_Pdev, bytes));
  if (harm_layout && !c->d_Paos) CK(cudaMalloc(&c->d_Paos, bytes));
  c->h_scal[0] = *dt;
  CK(cudaMemcpyAsync(c->d_dt, c->h_scal, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (stats) CK(cudaMemsetAsync(c->d_stats, 0, 5 * sizeof(double), c->stream));
  SlabWait sw;
  if (int rc = h2d_slabs(c, h_P, &sw, harm_layout)) return rc;
  if (enqueue_step(c, precision, guess, c->d_Pdev, stats != nullptr, &sw)) return 1;
  if (harm_layout) {
    if (hp_soa_to_harm(c, c->d_Pdev, c->d_Paos)) return 1;
    CK(cudaMemcpyAsync(h_P, c->d_Paos, bytes, cudaMemcpyDeviceToHost, c->stream));
  } else {
    CK(cudaMemcpyAsync(h_P, c->d_Pdev, bytes, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaMemcpyAsync(c->h_scal, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (stats) CK(cudaMemcpyAsync(c->h_scal + 8, c->d_stats, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (int rc = check_status(c)) return rc;
  *dt = c->h_scal[0];
  add_stats(c, stats, 2.0 * (double)d.n1 * d.n2 * d.n3, guess);
  return 0;
}

// D2H of the state d_Pdev into h_P in the slabs of h2d_slabs, on the D2H stream once the
// context stream's work so far (the step) is done; an event after each slab
static int d2h_slabs(harm_ctx* c, double* h_P) {
  if (!c->d2h_stream) {
    CK(cudaStreamCreateWithFlags(&c->d2h_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->done_ev, cudaEventDisableTiming));
    for (int s = 0; s < HARM_H2D_SLABS; s++) CK(cudaEventCreateWithFlags(&c->d2h_ev[s], cudaEventDisableTiming));
  }
  const int n3e = c->g.n3e;
  const int planes = (n3e + HARM_H2D_SLABS - 1) / HARM_H2D_SLABS;
  const int nslab = (n3e + planes - 1) / planes;
  CK(cudaEventRecord(c->done_ev, c->stream));
  CK(cudaStreamWaitEvent(c->d2h_stream, c->done_ev, 0));
  for (int s = 0; s < nslab; s++) {
    const int z0 = s * planes, z1 = (z0 + planes < n3e) ? z0 + planes : n3e;
    const size_t off = (size_t)z0 * c->plane, bytes = (size_t)(z1 - z0) * c->plane * sizeof(double);
    for (int p = 0; p < NPR; p++)
      CK(cudaMemcpyAsync(h_P + (size_t)p * c->cells + off, c->d_Pdev + (size_t)p * c->cells + off, bytes,
                         cudaMemcpyDeviceToHost, c->d2h_stream));
    CK(cudaEventRecord(c->d2h_ev[s], c->d2h_stream));
  }
  return 0;
}

// nsteps full steps over a host array, each step's state copied in from h_P and back out to
// it.  Step n's copy out runs in k-slabs on the D2H stream; step n+1's copy in of a slab waits
// only for the copy out of the same slab (the host values it reads), so the two PCIe
// directions overlap, and step n+1's first flux tiles start on the slabs already back.
extern "C" int harm_b200_step_host_n(harm_ctx* c, int precision, int guess, double* h_P, int nsteps, double* dt,
                                     harm_stats* stats) {
  if (!c || !h_P || !dt) return hb_setmsg("null argument", 1);
  if (nsteps < 1) return hb_setmsg("nsteps must be at least 1", 2);
  if (int rc = check_guess(c, guess)) return rc;
  if (int rc = check_precision(precision)) return rc;
  Dims d = dims_of(c->g);
  const size_t bytes = NPR * c->cells * sizeof(double);
  if (!c->d_Pdev) CK(cudaMalloc(&c->d_Pdev, bytes));
  c->h_scal[0] = *dt;
  CK(cudaMemcpyAsync(c->d_dt, c->h_scal, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (stats) CK(cudaMemsetAsync(c->d_stats, 0, 5 * sizeof(double), c->stream));
  for (int n = 0; n < nsteps; n++) {
    SlabWait sw;
    if (int rc = h2d_slabs(c, h_P, &sw, false, n > 0 ? c->d2h_ev : nullptr)) return rc;
    if (enqueue_step(c, precision, guess, c->d_Pdev, stats != nullptr, &sw)) return 1;
    if (int rc = d2h_slabs(c, h_P)) return rc;
  }
  CK(cudaMemcpyAsync(c->h_scal, c->d_dt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (stats) CK(cudaMemcpyAsync(c->h_scal + 8, c->d_stats, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaStreamSynchronize(c->d2h_stream));
  if (int rc = check_status(c)) return rc;
  *dt = c->h_scal[0];
  add_stats(c, stats, 2.0 * nsteps * (double)d.n1 * d.n2 * d.n3, guess);
  return 0;
}

extern "C" int harm_b200_step_host(harm_ctx* c, int precision, int guess, double* h_P, double* dt, harm_stats* stats) {
  return step_host(c, precision, guess, h_P, dt, stats, false);
}

extern "C" int harm_b200_step_host_harm(harm_ctx* c, int precision, int guess, double* h_P, double* dt,
                                        harm_stats* stats) {
  if (((uintptr_t)h_P % 16) != 0) return seterr_msg("the HARM-layout array must be 16-byte aligned", 2);
  return step_host(c, precision, guess, h_P, dt, stats, true);
}

extern "C" int harm_b200_utoprimgen_points(harm_ctx* c, size_t n, int guess, const double* d_U, const double* d_geom,
                                           double* d_P, int8_t* d_pflag, int32_t* d_iters) {
  if (int rc = check_guess(c, guess)) return rc;
  if (n == 0) return 0;
  if (hp_points(c, n, guess, d_U, d_geom, d_P, d_pflag, d_iters)) return 1;
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

namespace {
// CUDA events destroyed on every exit path of the function that holds them
struct StageEvents {
  cudaEvent_t ev[6];
  int made = 0;
  ~StageEvents() {
    for (int q = 0; q < made; q++) cudaEventDestroy(ev[q]);
  }
};
}  // namespace

// Stage times of one substep (substep 0 of the RK2 step on d_P; results into scratch).
extern "C" int harm_b200_time_stages(harm_ctx* c, int precision, int guess, const double* d_P, double dt, int reps,
                                     double* ms) {
  static const double CUf[4] = {1.0, 0.0, 0.5, 0.0};
  static const double Cun[4] = {0.0, 0.0, 0.0, 0.0};
  if (int rc = check_guess(c, guess)) return rc;
  if (int rc = check_precision(precision)) return rc;
  if (reps < 1) reps = 1;
  StageEvents se;
  cudaEvent_t* ev = se.ev;
  for (; se.made < 6; se.made++) CK(cudaEventCreate(&ev[se.made]));
  c->h_scal[0] = dt;
  CK(cudaMemcpyAsync(c->d_dt, c->h_scal, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  for (int q = 0; q < 5; q++) ms[q] = 0.0;
  StepCoef sc{};
  sc.CUf0 = CUf[0]; sc.CUf2 = CUf[2]; sc.Cun0 = Cun[0]; sc.Cun1 = Cun[1]; sc.Cun2 = Cun[2];
  sc.finalstep = 0; sc.guess = guess; sc.first = 1;
  for (int r = 0; r < reps; r++) {
    CK(cudaEventRecord(ev[0], c->stream));
    if (precision == HARM_PREC_FP64) {
      if (hp_fluxes_fp64(c, d_P, c->d_F[0], c->d_F[1], c->d_F[2], c->d_emf, c->d_dtslots)) return 1;
    } else if (precision == HARM_PREC_FP64_FMA) {
      if (hp_fluxes_fp64fma(c, d_P, c->d_F[0], c->d_F[1], c->d_F[2], c->d_emf, c->d_dtslots)) return 1;
    } else {
      if (hp_fluxes_mixed(c, d_P, c->d_Ff[0], c->d_Ff[1], c->d_Ff[2], c->d_emff, c->d_dtslots)) return 1;
    }
    CK(cudaEventRecord(ev[1], c->stream));
    CK(cudaEventRecord(ev[2], c->stream));
    if (precision == HARM_PREC_FP64) {
      if (hp_update_fp64(c, sc, d_P, d_P, c->d_pk, c->d_pflag, nullptr)) return 1;
    } else if (precision == HARM_PREC_FP64_FMA) {
      if (hp_update_fp64fma(c, sc, d_P, d_P, c->d_pk, c->d_pflag, nullptr)) return 1;
    } else {
      if (hp_update_mixed(c, sc, d_P, d_P, c->d_pk, c->d_pflag, nullptr)) return 1;
    }
    CK(cudaEventRecord(ev[3], c->stream));
    if (hp_bound(c, c->d_pk, nullptr)) return 1;
    CK(cudaEventRecord(ev[4], c->stream));
    if (hp_fixup(c, c->d_pk, c->d_pflag, 0)) return 1;
    CK(cudaEventRecord(ev[5], c->stream));
    CK(cudaEventSynchronize(ev[5]));
    float t;
    for (int q = 0; q < 5; q++) {
      CK(cudaEventElapsedTime(&t, ev[q], ev[q + 1]));
      ms[q] += t / reps;
    }
  }
  CK(cudaMemsetAsync(c->d_dtslots, 0xFF, 6 * sizeof(unsigned long long), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return check_status(c);
}
