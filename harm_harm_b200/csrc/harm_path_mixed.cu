// harm_path_mixed.cu -- mixed-precision path of the step: FP32 reconstruction, HLL and
// flux-CT; FP64 conserved update, sources and inversion (compiled with FMA contraction).
// the inversion of this path shares reciprocals between its FP64 divisions (harm_invert.cuh)
#define HARM_INVERT_FAST_DIV 1
// FP32 flux tiles at 3 resident blocks per SM (harm_common.cuh)
#ifndef HARM_FLUXT_MINB
#define HARM_FLUXT_MINB 3
#endif
#include <algorithm>
#include <cudaTypedefs.h>
#include <mutex>
#include "harm_common.cuh"
#include "harm_mlp_tc.cuh"
#include "harm_flux_tma.cuh"
#include "harm_paths.h"

int hb_setmsg(const char* msg, int code);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// whether the TMA-staged flux kernel can load this primitive array: 16-byte aligned base
// and row pitch (n1e even), and staging not switched off for the context
static bool tma_usable(const harm_ctx* c, const double* P) {
  return c->flux_tma && ((uintptr_t)P % 16 == 0) && (c->g.n1e % 2 == 0) && tensor_map_encoder() != nullptr;
}

// 4-D map of P[8][n3e][n2e][n1e] (FP64) with a box of bx x by x bz cells x 8 primitives
static int make_p_map(CUtensorMap* m, const double* P, const Dims& d, int bx, int by, int bz) {
  const cuuint64_t dims[4] = {(cuuint64_t)d.n1e, (cuuint64_t)d.n2e, (cuuint64_t)d.n3e, (cuuint64_t)NPR};
  const cuuint64_t strides[3] = {(cuuint64_t)d.n1e * 8, (cuuint64_t)d.n1e * d.n2e * 8, (cuuint64_t)d.cells * 8};
  const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz, (cuuint32_t)NPR};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = tensor_map_encoder()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(P), dims, strides, box, es,
                                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (r == CUDA_SUCCESS) ? 0 : hb_setmsg("cuTensorMapEncodeTiled failed for the primitive array", 4);
}

template <int DIR, int LIM>
static int launch_fluxt_tma(harm_ctx* c, const Dims& d, const Phys& ph, const FaceBox& fb, const double* P, float* F,
                            unsigned long long* slot) {
  using TB = TmaBox<DIR, LIM>;
  CUtensorMap map;
  if (int rc = make_p_map(&map, P, d, TB::BX, TB::BY, TB::BZ)) return rc;
  static std::atomic<unsigned long long> raised{0};  // per instantiation
  CK(raise_smem_limit_once(raised, (const void*)k_fluxt_tma<DIR, LIM, float>, (int)TB::smem));
  constexpr int A = FluxTile<LIM, float>::A, NT = FluxTile<LIM, float>::NT;
  const long long gx = (DIR == 1) ? (fb.cnt[0] + A - 1) / A : (fb.cnt[0] + NT - 1) / NT;
  const long long gy = (DIR == 1) ? (fb.cnt[1] + NT - 1) / NT : (DIR == 2) ? (fb.cnt[1] + A - 1) / A : (fb.cnt[2] + A - 1) / A;
  const long long gz = (DIR == 3) ? fb.cnt[1] : fb.cnt[2];
  const unsigned int nb = (unsigned int)std::min<long long>(gx * gy * gz, (long long)TmaOcc<LIM>::blocks * c->num_sms);
  k_fluxt_tma<DIR, LIM, float><<<nb, 256, TB::smem, c->stream>>>(d, ph, fb, map, c->d_geomf, F, slot, c->d_status);
  CK(cudaGetLastError());
  return 0;
}

template <int LIM>
static int flux_dirs_float(harm_ctx* c, const Dims& d, const Phys& ph, const double* pb, float* F1, float* F2, float* F3,
                         unsigned long long* slots, const SlabWait* sw) {
  // WENO5: the cell pass computes the dP line quantities once per cell for the three
  // directions (the plain-load tiles read them; the TMA-staged tiles compute their own)
  float* L = (LIM == HARM_LIM_WENO5) ? reinterpret_cast<float*>(c->d_line) : nullptr;
  if (sw) {  // state arriving in slabs: plain-load tiles, launched slab by slab
    CK((launch_flux_slabs<LIM, float, float>(d, ph, pb, c->d_geomf, F1, F2, F3, slots, c->stream, *sw, c->launches, L)));
    return 0;
  }
  FaceBox b1 = face_box(d, 1), b2 = face_box(d, 2), b3 = face_box(d, 3);
  // the TMA-staged variant covers MC, PARA and WENO5; PARALINE always takes k_fluxt
  if constexpr (LIM != HARM_LIM_PARALINE) {
    if (tma_usable(c, pb)) {
      if (int rc = launch_fluxt_tma<1, LIM>(c, d, ph, b1, pb, F1, slots + 0)) return rc;
      if (int rc = launch_fluxt_tma<2, LIM>(c, d, ph, b2, pb, F2, slots + 1)) return rc;
      c->launches += 2;
      if (d.n3 > 1) {
        if (int rc = launch_fluxt_tma<3, LIM>(c, d, ph, b3, pb, F3, slots + 2)) return rc;
        c->launches++;
      }
      return 0;
    }
  }
  if (L) {
    CK((launch_cellprep<float, float>(d, ph, pb, c->d_geomf, L, 0, d.n3e, c->stream)));
    c->launches++;
  }
  CK((launch_fluxt<1, LIM, float, float>(d, ph, b1, pb, c->d_geomf, F1, slots + 0, c->stream, L)));
  CK((launch_fluxt<2, LIM, float, float>(d, ph, b2, pb, c->d_geomf, F2, slots + 1, c->stream, L)));
  c->launches += 2;
  if (d.n3 > 1) {
    CK((launch_fluxt<3, LIM, float, float>(d, ph, b3, pb, c->d_geomf, F3, slots + 2, c->stream, L)));
    c->launches++;
  }
  return 0;
}

int hp_fluxes_mixed(harm_ctx* c, const double* pb, float* F1, float* F2, float* F3, float* emf,
                   unsigned long long* slots, const SlabWait* sw) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  if (c->g.lim == HARM_LIM_WENO5) { int rc = flux_dirs_float<HARM_LIM_WENO5>(c, d, ph, pb, F1, F2, F3, slots, sw); if (rc) return rc; }
  else if (c->g.lim == HARM_LIM_PARA) { int rc = flux_dirs_float<HARM_LIM_PARA>(c, d, ph, pb, F1, F2, F3, slots, sw); if (rc) return rc; }
  else if (c->g.lim == HARM_LIM_PARALINE) { int rc = flux_dirs_float<HARM_LIM_PARALINE>(c, d, ph, pb, F1, F2, F3, slots, sw); if (rc) return rc; }
  else { int rc = flux_dirs_float<HARM_LIM_MC>(c, d, ph, pb, F1, F2, F3, slots, sw); if (rc) return rc; }
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
  const CellTile ct = cell_tile(d.n3, HARM_INVERT_LTK);
  const CellTile cct = (HARM_CONSERVED_LTK > 0 && d.n3 >= 8) ? cell_tile(d.n3, HARM_CONSERVED_LTK) : cell_linear();
  if (ct.lti == 4) {  // 16 i x 16 k tiles: the metric and connection staged per block
    k_conserved_src<float, true><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(d, ph, sc, c->d_dt, pi, pb,
                                                                                        c->d_geom, c->d_conn, c->d_U, ct);
  } else {
    k_conserved_src<float, false><<<cell_grid(d.n1, d.n2, d.n3, cct), 256, 0, c->stream>>>(d, ph, sc, c->d_dt, pi, pb,
                                                                                          c->d_geom, c->d_conn, c->d_U, cct);
  }
  k_conserved_div<float><<<cell_grid(d.n1, d.n2, d.n3, cct), 256, 0, c->stream>>>(d, ph, sc, c->d_dt, c->d_Ff[0], c->d_Ff[1],
                                                                                 c->d_Ff[2], c->d_emff, c->d_U, cct);
  c->launches++;
  CK(cudaMemsetAsync(c->d_nrare, 0, sizeof(unsigned int), c->stream));
  if (sc.guess == HARM_GUESS_MLP && c->mlp_tc == 4) {
    if (int rc = launch_invert_gated<1>(c, d, ph, ct, pb, pf, pflag, stats)) return rc;
  } else if (sc.guess == HARM_GUESS_MLP && c->mlp_tc == 2) {
    if (int rc = launch_invert_tc<1>(c, d, ph, pb, pf, pflag, stats)) return rc;
  } else if (sc.guess == HARM_GUESS_MLP && c->mlp_tc == 3) {
    if (int rc = launch_invert_mma<1>(c, d, ph, ct, pb, pf, pflag, stats)) return rc;
  } else if (sc.guess == HARM_GUESS_MLP) {
    if (c->mlp_tc == 1) {
      if (int rc = launch_mlp_guess_tc<1>(c, d)) return rc;
    } else {
      k_mlp_guess<1><<<HARM_MLP_GUESS_BLOCKS * c->num_sms, 256, 0, c->stream>>>(d, c->d_U, c->d_geom, c->d_wpg,
                                                      reinterpret_cast<const MlpPacked*>(c->d_mlp), ct);
      c->launches++;
    }
    k_invert<1, true><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag,
                                                          c->d_geom, c->d_aux, c->d_rare, c->d_nrare, stats, ct, c->d_wpg);
    c->launches++;
  } else {
    k_invert<1><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag, c->d_geom,
                                                    c->d_aux, c->d_rare, c->d_nrare, stats, ct);
    c->launches++;
  }
  k_invert_rare<1><<<2 * c->num_sms, 128, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag, c->d_geom, c->d_aux, c->d_rare,
                                                     c->d_nrare, stats);
  c->launches += 2;
  CK(cudaGetLastError());
  return 0;
}

// The reciprocal of this path's inversion (frcp, harm_invert.cuh) over n device values, so
// that its error against IEEE division can be checked over the operand range.
__global__ void k_mixed_reciprocal(const double* __restrict__ b, double* __restrict__ r, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    r[i] = frcp(b[i]);
}

extern "C" int harm_b200_mixed_reciprocal(harm_ctx* c, const double* d_b, double* d_r, size_t n) {
  if (!c || (n && (!d_b || !d_r))) return hb_setmsg("null argument", 1);
  if (n == 0) return 0;
  const size_t blocks = std::min<size_t>((n + 255) / 256, (size_t)4 * (c->num_sms > 0 ? c->num_sms : 1));
  k_mixed_reciprocal<<<(unsigned)blocks, 256, 0, c->stream>>>(d_b, d_r, n);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}
