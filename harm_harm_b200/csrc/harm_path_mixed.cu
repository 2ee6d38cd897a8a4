// harm_path_mixed.cu -- mixed-precision path of the step: FP32 reconstruction, HLL and
// flux-CT; FP64 conserved update, sources and inversion (compiled with FMA contraction).
#include "harm_common.cuh"
#include "harm_paths.h"

template <int LIM>
static int flux_dirs_float(harm_ctx* c, const Dims& d, const Phys& ph, const double* pb, float* F1, float* F2, float* F3,
                         unsigned long long* slots) {
  FaceBox b1 = face_box(d, 1), b2 = face_box(d, 2), b3 = face_box(d, 3);
  CK((launch_fluxt<1, LIM, float, float>(d, ph, b1, pb, c->d_geomf, F1, slots + 0, c->stream)));
  CK((launch_fluxt<2, LIM, float, float>(d, ph, b2, pb, c->d_geomf, F2, slots + 1, c->stream)));
  c->launches += 2;
  if (d.n3 > 1) {
    CK((launch_fluxt<3, LIM, float, float>(d, ph, b3, pb, c->d_geomf, F3, slots + 2, c->stream)));
    c->launches++;
  }
  return 0;
}

int hp_fluxes_mixed(harm_ctx* c, const double* pb, float* F1, float* F2, float* F3, float* emf,
                   unsigned long long* slots) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  if (c->g.lim == HARM_LIM_WENO5) { int rc = flux_dirs_float<HARM_LIM_WENO5>(c, d, ph, pb, F1, F2, F3, slots); if (rc) return rc; }
  else if (c->g.lim == HARM_LIM_PARA) { int rc = flux_dirs_float<HARM_LIM_PARA>(c, d, ph, pb, F1, F2, F3, slots); if (rc) return rc; }
  else { int rc = flux_dirs_float<HARM_LIM_MC>(c, d, ph, pb, F1, F2, F3, slots); if (rc) return rc; }
  long long nc = (long long)(d.n1 + 1) * (d.n2 + 1) * (d.n3 > 1 ? d.n3 + 1 : 1);
  k_emf<float, float><<<nblk(nc), 256, 0, c->stream>>>(d, F1, F2, F3, c->d_geomf, emf);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

int hp_update_mixed(harm_ctx* c, const StepCoef& sc, const double* pi, const double* pb, double* pf, int8_t* pflag,
                    double* stats) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  long long ncell = (long long)d.n1 * d.n2 * d.n3;
  (void)ncell;
  const CellTile ct = cell_tile(d.n3);
  k_conserved<float><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(d, ph, sc, c->d_dt, pi, pb, c->d_Ff[0], c->d_Ff[1],
                                                         c->d_Ff[2], c->d_emff, c->d_geom, c->d_conn, c->d_U, ct);
  CK(cudaMemsetAsync(c->d_nrare, 0, sizeof(unsigned int), c->stream));
  if (sc.guess == HARM_GUESS_MLP) {
    k_mlp_guess<1><<<3 * 148, 256, 0, c->stream>>>(d, c->d_U, c->d_geom, c->d_wpg,
                                                    reinterpret_cast<const MlpPacked*>(c->d_mlp), ct);
    k_invert<1, true><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag,
                                                          c->d_geom, c->d_aux, c->d_rare, c->d_nrare, stats, ct, c->d_wpg);
    c->launches++;
  } else {
    k_invert<1><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag, c->d_geom,
                                                    c->d_aux, c->d_rare, c->d_nrare, stats, ct);
  }
  k_invert_rare<1><<<2 * 148, 128, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag, c->d_geom, c->d_aux, c->d_rare,
                                                     c->d_nrare, stats);
  c->launches += 3;
  CK(cudaGetLastError());
  return 0;
}
