// harm_noalloc_fp64.cu -- fluxcalc for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they need the fluxes: code that
// runs inside a memory pool or arena it does not own, an embedding host that forbids
// allocation during its time loop, or a driver that must not grow the device footprint
// after start-up.  harm_b200_fluxcalc_noalloc gives them the same FP64 fluxes as
// harm_b200_fluxcalc without allocating anything: the caller passes the metric table,
// the primitives and the three flux arrays, and the EMF scratch of flux-CT and the CFL
// minima live in file-scope __device__ arrays of fixed size, which every GPU that loads
// the library holds until the process exits.
//
// Limits and behaviour:
//   - at most HARM_NOALLOC_MAX_CELLS extended cells (n1e*n2e*n3e); larger grids are
//     rejected with an error before any work is queued;
//   - every call shares the same scratch, which keeps the last call's contents; the CFL
//     minima are reset at the start of each call and the EMFs are fully rewritten, so a
//     call never reads what an earlier call left behind;
//   - calls that overlap on the GPU (concurrent streams, or several host threads) race on
//     the shared scratch and must be serialised by the caller;
//   - the first call on a device looks up the device address of the scratch with
//     cudaGetSymbolAddress (with that device current) and caches it;
//   - the call is synchronous: it copies the CFL minima back to the host and waits for its
//     own stream before returning ndt.
// The kernels are the FP64 path's, compiled the same way (no FMA contraction), so the
// results equal harm_b200_fluxcalc's.
#ifndef HARM_FLUXT_MINB
#define HARM_FLUXT_MINB 2  // the FP64 flux tiles at 2 blocks per SM, as in harm_path_fp64.cu
#endif
#include <mutex>
#include "harm_common.cuh"

static __device__ __align__(256) double g_noalloc_emf[3 * (size_t)HARM_NOALLOC_MAX_CELLS];
static __device__ __align__(256) unsigned long long g_noalloc_dtmin[4];

static std::mutex g_noalloc_mu;
static double* g_noalloc_emf_ptr[64];
static unsigned long long* g_noalloc_dt_ptr[64];

// error text goes to the library's harm_b200_last_error() buffer
int hb_setmsg(const char* msg, int code);

static int noalloc_fail(const char* msg) {
  char buf[256];
  snprintf(buf, sizeof(buf), "harm_b200_fluxcalc_noalloc: %s", msg);
  return hb_setmsg(buf, 1);
}

// Device addresses of the scratch arrays for the current device (looked up once per device).
static int noalloc_scratch(double** emf, unsigned long long** dtmin) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return noalloc_fail("cudaGetDevice failed");
  if (dev < 0 || dev >= 64) return noalloc_fail("device index out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_emf_ptr[dev]) {
    void* pe = nullptr;
    void* pd = nullptr;
    cudaError_t e1 = cudaGetSymbolAddress(&pe, g_noalloc_emf);
    if (e1 != cudaSuccess) return noalloc_fail(cudaGetErrorString(e1));
    cudaError_t e2 = cudaGetSymbolAddress(&pd, g_noalloc_dtmin);
    if (e2 != cudaSuccess) return noalloc_fail(cudaGetErrorString(e2));
    g_noalloc_emf_ptr[dev] = (double*)pe;
    g_noalloc_dt_ptr[dev] = (unsigned long long*)pd;
  }
  *emf = g_noalloc_emf_ptr[dev];
  *dtmin = g_noalloc_dt_ptr[dev];
  return 0;
}

// the three directions with the FP64 path's tile kernel (the first launch of an instantiation
// on a device raises its shared-memory limit where the tile needs more than 48 KB)
template <int LIM>
static cudaError_t noalloc_dirs(const Dims& d, const Phys& ph, const double* geom, const double* pb, double* F1,
                                double* F2, double* F3, unsigned long long* dtmin, cudaStream_t st) {
  cudaError_t e = launch_fluxt<1, LIM, double, double>(d, ph, face_box(d, 1), pb, geom, F1, dtmin + 0, st);
  if (e == cudaSuccess) e = launch_fluxt<2, LIM, double, double>(d, ph, face_box(d, 2), pb, geom, F2, dtmin + 1, st);
  if (e == cudaSuccess && d.n3 > 1) e = launch_fluxt<3, LIM, double, double>(d, ph, face_box(d, 3), pb, geom, F3, dtmin + 2, st);
  return e;
}

extern "C" int harm_b200_fluxcalc_noalloc(const harm_grid* g, const double* d_geom, const double* d_pb, double* d_F1,
                                          double* d_F2, double* d_F3, double ndt[3], void* stream) {
  if (!g || !d_geom || !d_pb || !d_F1 || !d_F2 || !d_F3 || !ndt) return noalloc_fail("null argument");
  if (g->lim != HARM_LIM_MC && g->lim != HARM_LIM_PARA && g->lim != HARM_LIM_WENO5 && g->lim != HARM_LIM_PARALINE)
    return noalloc_fail("unknown reconstruction");
  if ((g->lim == HARM_LIM_WENO5 && g->ng < 6) || g->ng < 4) return noalloc_fail("too few ghost zones for the reconstruction");
  const size_t cells = (size_t)g->n1e * g->n2e * g->n3e;
  if (cells > (size_t)HARM_NOALLOC_MAX_CELLS) {
    char buf[256];
    snprintf(buf, sizeof(buf), "harm_b200_fluxcalc_noalloc: grid has %zu extended cells, the maximum is %d", cells,
             (int)HARM_NOALLOC_MAX_CELLS);
    return hb_setmsg(buf, 2);
  }
  double* emf;
  unsigned long long* dtmin;
  if (noalloc_scratch(&emf, &dtmin)) return 1;
  cudaStream_t st = (cudaStream_t)stream;
  Dims d = dims_of(*g);
  Phys ph = phys_of(*g);
  // the CFL minima start from the identity of the min reduction
  if (cudaMemsetAsync(dtmin, 0xFF, 3 * sizeof(unsigned long long), st) != cudaSuccess)
    return noalloc_fail("cudaMemsetAsync failed");
  cudaError_t e;
  if (g->lim == HARM_LIM_WENO5) e = noalloc_dirs<HARM_LIM_WENO5>(d, ph, d_geom, d_pb, d_F1, d_F2, d_F3, dtmin, st);
  else if (g->lim == HARM_LIM_PARA) e = noalloc_dirs<HARM_LIM_PARA>(d, ph, d_geom, d_pb, d_F1, d_F2, d_F3, dtmin, st);
  else if (g->lim == HARM_LIM_PARALINE) e = noalloc_dirs<HARM_LIM_PARALINE>(d, ph, d_geom, d_pb, d_F1, d_F2, d_F3, dtmin, st);
  else e = noalloc_dirs<HARM_LIM_MC>(d, ph, d_geom, d_pb, d_F1, d_F2, d_F3, dtmin, st);
  if (e != cudaSuccess) return noalloc_fail(cudaGetErrorString(e));
  long long nc = (long long)(d.n1 + 1) * (d.n2 + 1) * (d.n3 > 1 ? d.n3 + 1 : 1);
  k_emf<double, double><<<nblk(nc), 256, 0, st>>>(d, d_F1, d_F2, d_F3, d_geom, emf);
  k_emf_to_flux<double><<<nblk(nc), 256, 0, st>>>(d, emf, d_F1, d_F2, d_F3);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(cudaGetErrorString(e));
  unsigned long long hb[3];
  if (cudaMemcpyAsync(hb, dtmin, sizeof(hb), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return noalloc_fail("cudaMemcpyAsync failed");
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return noalloc_fail(cudaGetErrorString(e));
  for (int q = 0; q < 3; q++) {
    double v;
    memcpy(&v, &hb[q], 8);
    ndt[q] = (hb[q] == 0xFFFFFFFFFFFFFFFFull) ? 1.e100 : v;
  }
  return 0;
}
