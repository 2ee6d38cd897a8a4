// harm_layout.cu -- HARM's own array layout at the C ABI.
//
// HARM stores its primitive, conserved and flux arrays as FTYPE [N3M][N2M][N1M][NPR]
// (ORDERSTORAGE 5, global.storage.h:320-340: the eight values of a cell together, i fastest
// among cells) and its failure flags as PFTYPE (signed int) [N3M][N2M][N1M][NUMPFLAGS].  The
// device kernels keep one array per primitive, [pl][k][j][i], so that a warp's loads of one
// primitive along i are coalesced.  These entry points convert between the two on the device
// (over the extended grid, ghost zones included: HARM's MAXBND must equal the grid's ng), and
// harm_b200_step_host_harm runs one step over a host array in HARM's layout, the conversion
// of each arriving k-slab ahead of the first flux tiles that stage it.
#include "harm_common.cuh"
#include "harm_paths.h"

int hb_setmsg(const char* msg, int code);

// [k][j][i][pl] -> [pl][k][j][i] for the cells of planes [k0, k1): a thread per cell, the
// cell's 64 bytes read as four 16-byte loads (a warp reads 2 KB contiguous), one coalesced
// store per primitive
__global__ void __launch_bounds__(256) k_harm_to_soa(Dims d, const double* __restrict__ aos, double* __restrict__ soa,
                                                     int k0, int k1) {
  const long long n = (long long)(k1 - k0) * d.plane;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const size_t id = (size_t)k0 * d.plane + (size_t)t;
  const double2* src = reinterpret_cast<const double2*>(aos + (size_t)NPR * id);
#pragma unroll
  for (int q = 0; q < NPR / 2; q++) {
    const double2 v = __ldg(src + q);
    soa[(size_t)(2 * q) * d.cells + id] = v.x;
    soa[(size_t)(2 * q + 1) * d.cells + id] = v.y;
  }
}

__global__ void __launch_bounds__(256) k_soa_to_harm(Dims d, const double* __restrict__ soa, double* __restrict__ aos,
                                                     int k0, int k1) {
  const long long n = (long long)(k1 - k0) * d.plane;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const size_t id = (size_t)k0 * d.plane + (size_t)t;
  double2* dst = reinterpret_cast<double2*>(aos + (size_t)NPR * id);
#pragma unroll
  for (int q = 0; q < NPR / 2; q++)
    dst[q] = make_double2(__ldg(soa + (size_t)(2 * q) * d.cells + id), __ldg(soa + (size_t)(2 * q + 1) * d.cells + id));
}

// flag slot 0 (FLAGUTOPRIMFAIL) of HARM's [cell][numpflags] ints <-> the device's int8 per cell
__global__ void k_flags_to_harm(size_t cells, const int8_t* __restrict__ f, int32_t* __restrict__ hf, int numpflags) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < cells) hf[t * (size_t)numpflags] = (int32_t)f[t];
}
__global__ void k_flags_from_harm(size_t cells, const int32_t* __restrict__ hf, int8_t* __restrict__ f, int numpflags) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < cells) f[t] = (int8_t)hf[t * (size_t)numpflags];
}

static unsigned int blocks_of(long long n) { return (unsigned int)((n + 255) / 256); }

int hp_harm_to_soa(harm_ctx* c, const double* aos, double* soa, int k0, int k1) {
  const Dims d = dims_of(c->g);
  const long long n = (long long)(k1 - k0) * d.plane;
  if (n <= 0) return 0;
  k_harm_to_soa<<<blocks_of(n), 256, 0, c->stream>>>(d, aos, soa, k0, k1);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

static int aligned16(const void* p) { return ((uintptr_t)p % 16) == 0; }

extern "C" int harm_b200_from_harm_layout(harm_ctx* c, const double* d_harm, double* d_P) {
  if (!c || !d_harm || !d_P) return hb_setmsg("null argument", 1);
  if (!aligned16(d_harm)) return hb_setmsg("the HARM-layout array must be 16-byte aligned", 2);
  return hp_harm_to_soa(c, d_harm, d_P, 0, c->g.n3e);
}

extern "C" int harm_b200_to_harm_layout(harm_ctx* c, const double* d_P, double* d_harm) {
  if (!c || !d_harm || !d_P) return hb_setmsg("null argument", 1);
  if (!aligned16(d_harm)) return hb_setmsg("the HARM-layout array must be 16-byte aligned", 2);
  const Dims d = dims_of(c->g);
  k_soa_to_harm<<<blocks_of((long long)d.cells), 256, 0, c->stream>>>(d, d_P, d_harm, 0, d.n3e);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

extern "C" int harm_b200_flags_to_harm(harm_ctx* c, const int8_t* d_pflag, int32_t* d_harm_pflag, int numpflags) {
  if (!c || !d_pflag || !d_harm_pflag) return hb_setmsg("null argument", 1);
  if (numpflags < 1) return hb_setmsg("numpflags must be at least 1", 2);
  k_flags_to_harm<<<blocks_of((long long)c->cells), 256, 0, c->stream>>>(c->cells, d_pflag, d_harm_pflag, numpflags);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

extern "C" int harm_b200_flags_from_harm(harm_ctx* c, const int32_t* d_harm_pflag, int8_t* d_pflag, int numpflags) {
  if (!c || !d_pflag || !d_harm_pflag) return hb_setmsg("null argument", 1);
  if (numpflags < 1) return hb_setmsg("numpflags must be at least 1", 2);
  k_flags_from_harm<<<blocks_of((long long)c->cells), 256, 0, c->stream>>>(c->cells, d_harm_pflag, d_pflag, numpflags);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

int hp_soa_to_harm(harm_ctx* c, const double* soa, double* aos) {
  const Dims d = dims_of(c->g);
  k_soa_to_harm<<<blocks_of((long long)d.cells), 256, 0, c->stream>>>(d, soa, aos, 0, d.n3e);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}
