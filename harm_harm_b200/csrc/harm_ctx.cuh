// harm_ctx.cuh -- device context of libharm_b200.so (opaque to callers).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "harm_b200.h"

// the host-buffer entry point copies the state in k-slabs: at most this many, each followed by
// an event the first substep's flux launches of that slab wait for
#define HARM_H2D_SLABS 8

struct harm_ctx;

// which copy event each k-plane's flux launches wait for (planes [s*planes, (s+1)*planes) of
// the extended grid arrive with ev[s]); with aos set, the slabs arrive in HARM's
// [k][j][i][pl] layout there and are converted into soa after their event
struct SlabWait {
  const cudaEvent_t* ev;
  int nslab, planes;
  harm_ctx* ctx;
  const double* aos;
  double* soa;
};

struct harm_ctx {
  harm_grid g;
  int device;
  cudaStream_t stream;
  cudaStream_t copy_stream;             // host-buffer entry point: H2D of the state
  cudaEvent_t slab_ev[HARM_H2D_SLABS];  // recorded on copy_stream after each slab
  cudaEvent_t entry_ev;                 // recorded on stream before the copies start
  cudaStream_t d2h_stream;              // multi-step host-buffer entry point: D2H of the state
  cudaEvent_t d2h_ev[HARM_H2D_SLABS];   // recorded on d2h_stream after each slab
  cudaEvent_t done_ev;                  // recorded on stream when a step's state is final
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
  void* d_line;     // WENO5: dP line quantities of the flux stage's cell pass, [9][cells] (FP64
                    // path: double, mixed path: float)
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
  double* d_Paos;   // the same in HARM's [k][j][i][pl] layout (harm_b200_step_host_harm)
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
  int mlp_tc;              // learned start: 4 gated (default: the network, fused with the
                           // inversion, only for cells whose previous state is a poor start),
                           // or for every cell: 0 mma.sync network kernel ahead of the
                           // inversion (HARM_B200_MLP_ENGINE=mma), 1 tcgen05 network kernel
                           // ahead of it (=tc), 2 tcgen05 inside the inversion kernel
                           // (=tc-fused), 3 mma.sync inside the inversion kernel (=mma-fused)
  double mlp_gate;         // gated engine: a first Newton step above this fraction of the
                           // convergence scale marks a poor previous-state start
                           // (HARM_B200_MLP_GATE, default 0.02)
  unsigned int* d_nhard;   // gated engine: length of its list of poorly started cells
  int num_sms;
  unsigned long long launches;  // kernels launched by this context
};
