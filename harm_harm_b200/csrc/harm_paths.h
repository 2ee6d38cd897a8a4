// harm_paths.h -- launch entry points of the two arithmetic paths (host side).
#pragma once
#include <stdint.h>
#include "harm_ctx.cuh"

struct StepCoef;

// fluxes and EMFs of one substep; sw: the state is still arriving in k-slabs (launches wait
// for each slab's copy event)
int hp_fluxes_fp64(harm_ctx* c, const double* pb, double* F1, double* F2, double* F3, double* emf,
                   unsigned long long* slots, const SlabWait* sw = nullptr);
int hp_fluxes_mixed(harm_ctx* c, const double* pb, float* F1, float* F2, float* F3, float* emf,
                    unsigned long long* slots, const SlabWait* sw = nullptr);
int hp_update_fp64(harm_ctx* c, const StepCoef& sc, const double* pi, const double* pb, double* pf, int8_t* pflag,
                   double* stats);
// the same, compiled with FMA contraction (harm_path_fp64fma.cu)
int hp_fluxes_fp64fma(harm_ctx* c, const double* pb, double* F1, double* F2, double* F3, double* emf,
                      unsigned long long* slots, const SlabWait* sw = nullptr);
int hp_update_fp64fma(harm_ctx* c, const StepCoef& sc, const double* pi, const double* pb, double* pf,
                      int8_t* pflag, double* stats);
int hp_update_mixed(harm_ctx* c, const StepCoef& sc, const double* pi, const double* pb, double* pf, int8_t* pflag,
                    double* stats);
int hp_emf_to_flux_fp64(harm_ctx* c, const double* emf, double* F1, double* F2, double* F3);
int hp_bound(harm_ctx* c, double* P, int8_t* flag);
int hp_copy_ghosts(harm_ctx* c, const double* pb, double* pf);
// post_fixup of the final substep (finalstep 1) or an earlier one (0); bound_flags = false when
// the caller has already filled the flags' ghost zones
int hp_fixup(harm_ctx* c, double* pf, int8_t* pflag, int finalstep, bool bound_flags = true);
int hp_finalize_dt(harm_ctx* c, double* dt, double* ndt_out, int nsub);
int hp_points(harm_ctx* c, size_t n, int guess, const double* U, const double* geom, double* P, int8_t* pflag, int32_t* iters);
// the metric, connection and floor tables computed on the device; their FP32 copy
int hp_geometry_build(harm_ctx* c);
int hp_geometry_f32(harm_ctx* c);
// HARM's [k][j][i][pl] layout <-> the device's [pl][k][j][i] (harm_layout.cu): planes [k0, k1)
int hp_harm_to_soa(harm_ctx* c, const double* aos, double* soa, int k0, int k1);
int hp_soa_to_harm(harm_ctx* c, const double* soa, double* aos);
