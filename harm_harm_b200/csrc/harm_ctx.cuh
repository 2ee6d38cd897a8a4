// harm_ctx.cuh -- device context of libharm_b200.so (opaque to callers).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "harm_b200.h"

// the host-buffer entry point copies the state in k-slabs: at most this many, each followed by
// an event the first substep's flux launches of that slab wait for
#define HARM_H2D_SLABS 8

// which copy event each k-plane's flux launches wait for (planes [s*planes, (s+1)*planes) of
// the extended grid arrive with ev[s])
struct SlabWait {
  const cudaEvent_t* ev;
  int nslab, planes;
};

struct harm_ctx {
  harm_grid g;
  int device;
  cudaStream_t stream;
  cudaStream_t copy_stream;             // host-buffer entry point: H2D of the state
  cudaEvent_t slab_ev[HARM_H2D_SLABS];  // recorded on copy_stream after each slab
  cudaEvent_t entry_ev;                 // recorded on stream before the copies start
  size_t plane, cells;
  // metric tables (FP64, plus an FP32 copy for the mixed-precision flux path)
  double* d_geom;
  float* d_geomf;
  double* d_conn;
  double* d_aux;
  // scratch of one substep
  double* d_F[3];
  float* d_Ff[3];
  double* d_emf;
  float* d_emff;
  double* d_pk;     // midpoint primitives of the RK2 step
  double* d_U;      // conserved variables to invert (UEVOLVE)
  unsigned int* d_rare;   // cells finished by the rare inversion path
  unsigned int* d_nrare;  // their count
  int8_t* d_pflag;  // inversion flags
  void* d_fixrec;   // fixup records
  unsigned int fix_cap;
  // device scalars: dt slots, dt, ndt, stats, fixup counter
  double* d_scal;
  unsigned long long* d_dtslots;
  double* d_dt;
  double* d_ndt;
  double* d_stats;
  unsigned int* d_nrec;
  double* h_scal;   // pinned host mirror
  double* d_Pdev;   // device state used by the host-buffer entry point
  // learned guess
  float* d_mlp;        // inference records (MlpPacked for mma.sync, then MlpTc for tcgen05)
  double* d_wpg;       // learned starting W' of each active cell (k_mlp_guess)
  float* d_mlp_master; // FP32 master parameters
  float* d_mlp_adam;   // Adam moments
  float* d_mlp_work;   // training workspace
  size_t mlp_work_n;
  int mlp_step;
  unsigned int* d_status; // device error word (bit 0: a TMA tile wait timed out, bit 1: a
                          // tensor-core MMA wait of the learned start timed out)
  int flux_tma;            // stage the FP32 flux tiles with TMA (HARM_B200_FLUX_STAGING=tma)
  int mlp_tc;              // learned start: 0 mma.sync network kernel ahead of the inversion
                           // (default), 1 tcgen05 network kernel ahead of it
                           // (HARM_B200_MLP_ENGINE=tc), 2 tcgen05 inside the inversion
                           // kernel (=tc-fused), 3 mma.sync inside the inversion kernel
                           // (=mma-fused)
  int num_sms;
  unsigned long long launches;  // kernels launched by this context
};
