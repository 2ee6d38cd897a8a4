// harm_mlp_data_fp64.cu -- training pairs of the learned inversion guess.
//
// Two producers of (features, targets) pairs, both on the device:
//   - the grid dump: the conserved state of the context's most recent inversion (the U the
//     plain method inverted in its own run) and the primitives that came out of it; the
//     target is the converged W' of a Newton re-solve (plain guess), so cells where the
//     hot inversion fails are left out;
//   - synthetic states: primitives drawn from wide distributions (rho log-uniform in
//     [1e-6, 1], u/rho log-uniform in [1e-4, 1e2], gamma uniform in [1, 50], b^2/rho
//     log-uniform in [1e-3, 1e3], isotropic directions in the cell's coordinate frame
//     normalised by sqrt(g_ii)), at Boyer-Lindquist r uniform in [1.2, 40] (clamped to the
//     grid) and a uniformly drawn x2 row of the context's metric table; U from the
//     device primtoU, the targets from the drawn primitives.
// Features and targets are those of harm_mlp.cuh.  Compiled without FMA contraction, like
// the FP64 path, so the FP64 feature arithmetic is the oracle's.
#include <algorithm>
#include "harm_common.cuh"
#include "harm_mlp.cuh"

int hb_setmsg(const char* msg, int code);

namespace {

__device__ __forceinline__ uint64_t smix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// uniform in [0,1): draw k of sample i
__device__ __forceinline__ double urand(uint64_t seed, uint64_t i, int k) {
  return (double)(smix(seed ^ smix(i * 16ull + (uint64_t)k)) >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void k_mlp_dump(Dims d, Phys ph, const double* __restrict__ U, const double* __restrict__ P,
                           const double* __restrict__ geom, int stride, int phase, unsigned int max,
                           float* __restrict__ feat, float* __restrict__ targ, int32_t* __restrict__ cell,
                           unsigned int* __restrict__ count) {
  const long long ncell = (long long)d.n1 * d.n2 * d.n3;
  const long long nsel = (ncell - phase + stride - 1) / stride;
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nsel) return;
  long long t = phase + k * stride;
  int i = (int)(t % d.n1);
  long long r = t / d.n1;
  int j = (int)(r % d.n2), kk = (int)(r / d.n2);
  int ii = i + d.ng, jj = j + d.ng, k3 = kk + d.ng3;
  const size_t id = cidx(d, ii, jj, k3), c2 = (size_t)jj * d.n1e + ii;
  Geo<double> g;
  load_geo<double, double>(geom, d.plane, c2, g);
  double Ugf[NPR], pr[NPR];
#pragma unroll
  for (int p = 0; p < NPR; p++) { Ugf[p] = U[(size_t)p * d.cells + id] * g.igdet; pr[p] = P[(size_t)p * d.cells + id]; }
  JonSetup s;
  jon_prepare(false, Ugf, g, pr, ph.gam, ph.gammafail, s);
  float f[MLP_IN], tg[MLP_OUT];
  mlp_features(s.c, g, f);
  int8_t flag = 0;
  int it = 0;
  double wp = 0.0;
  jon_solve(s, s.Wp_prev, pr, flag, it, &wp);
  if (flag != 0 || !isfinite(wp)) return;
  mlp_targets(wp, s.c, tg);
  unsigned int slot = atomicAdd(count, 1u);
  if (slot >= max) return;
#pragma unroll
  for (int q = 0; q < MLP_IN; q++) feat[(size_t)slot * MLP_IN + q] = f[q];
#pragma unroll
  for (int q = 0; q < MLP_OUT; q++) targ[(size_t)slot * MLP_OUT + q] = tg[q];
  if (cell) cell[slot] = (int32_t)t;
}

// a direction drawn isotropically, scaled by 1/sqrt(g_ii) per coordinate
__device__ __forceinline__ void draw_dir(uint64_t seed, uint64_t t, int k0, const Geo<double>& g, double* v) {
  const double z = 2.0 * urand(seed, t, k0) - 1.0, ph = 6.283185307179586 * urand(seed, t, k0 + 1);
  const double s = sqrt(fmax(0.0, 1.0 - z * z));
  v[0] = s * cos(ph) / sqrt(g.gcov[4]);
  v[1] = s * sin(ph) / sqrt(g.gcov[7]);
  v[2] = z / sqrt(g.gcov[9]);
}

__global__ void k_mlp_synth(Dims d, Phys ph, size_t n, uint64_t seed, const double* __restrict__ geom,
                            const double* __restrict__ aux, float* __restrict__ feat, float* __restrict__ targ,
                            double* __restrict__ Uout, double* __restrict__ Pout, int32_t* __restrict__ cell) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  // cell: x2 row uniform, then the x1 index whose r is the largest not above the drawn r
  int j = min((int)(urand(seed, t, 0) * d.n2), d.n2 - 1);
  const int jj = j + d.ng;
  const double rt = 1.2 + (40.0 - 1.2) * urand(seed, t, 1);
  const double* R = aux + (size_t)HARM_AUX_R * d.plane + (size_t)jj * d.n1e + d.ng;
  int lo = 0, hi = d.n1 - 1;
  if (R[0] >= rt) hi = 0;
  while (lo < hi) {  // largest i with R[i] <= rt
    int mid = (lo + hi + 1) >> 1;
    if (R[mid] <= rt) lo = mid; else hi = mid - 1;
  }
  const int ii = lo + d.ng;
  const size_t c2 = (size_t)jj * d.n1e + ii;
  Geo<double> g;
  load_geo<double, double>(geom, d.plane, c2, g);
  double pr[NPR];
  const double rho = pow(10.0, -6.0 + 6.0 * urand(seed, t, 2));
  const double u = rho * pow(10.0, -4.0 + 6.0 * urand(seed, t, 3));
  const double gamma = 1.0 + 49.0 * urand(seed, t, 4);
  const double sigma = pow(10.0, -3.0 + 6.0 * urand(seed, t, 5));
  double v[3], e[3];
  draw_dir(seed, t, 6, g, v);
  draw_dir(seed, t, 8, g, e);
  pr[HARM_RHO] = rho;
  pr[HARM_UU] = u;
  pr[HARM_U1] = v[0]; pr[HARM_U2] = v[1]; pr[HARM_U3] = v[2];
  pr[HARM_B1] = 0.0; pr[HARM_B2] = 0.0; pr[HARM_B3] = 0.0;
  const double q0 = qsq_of<double>(pr, g);
  const double sc = (q0 > 0.0) ? sqrt((gamma * gamma - 1.0) / q0) : 0.0;
  pr[HARM_U1] *= sc; pr[HARM_U2] *= sc; pr[HARM_U3] *= sc;
  pr[HARM_B1] = e[0]; pr[HARM_B2] = e[1]; pr[HARM_B3] = e[2];
  State<double> q;
  get_state<double>(pr, g, ph.gam, q);
  const double bsc = (q.bsq > 0.0) ? sqrt(sigma * rho / q.bsq) : 0.0;
  pr[HARM_B1] *= bsc; pr[HARM_B2] *= bsc; pr[HARM_B3] *= bsc;
  get_state<double>(pr, g, ph.gam, q);
  double Ug[NPR];
  primtoflux<double>(pr, q, 0, g, g.gdet, Ug);
  // features from U exactly as the inversion sees it; targets from the drawn primitives
  double Ugf[NPR], prc[NPR];
#pragma unroll
  for (int p = 0; p < NPR; p++) { Ugf[p] = Ug[p] * g.igdet; prc[p] = pr[p]; }
  JonSetup s;
  jon_prepare(false, Ugf, g, prc, ph.gam, ph.gammafail, s);
  float f[MLP_IN], tg[MLP_OUT];
  mlp_features(s.c, g, f);
  const double utsq = q.qsq, gm = sqrt(1.0 + utsq), pgas = (ph.gam - 1.0) * u;
  const double wp = s.c.D * utsq / (1.0 + gm) + (u + pgas) * (1.0 + utsq);
  mlp_targets(wp, s.c, tg);
#pragma unroll
  for (int p = 0; p < MLP_IN; p++) feat[t * MLP_IN + p] = f[p];
#pragma unroll
  for (int p = 0; p < MLP_OUT; p++) targ[t * MLP_OUT + p] = tg[p];
  if (Uout) {
#pragma unroll
    for (int p = 0; p < NPR; p++) Uout[(size_t)p * n + t] = Ug[p];
  }
  if (Pout) {
#pragma unroll
    for (int p = 0; p < NPR; p++) Pout[(size_t)p * n + t] = pr[p];
  }
  if (cell) cell[t] = (int32_t)c2;
}

}  // namespace

extern "C" int harm_b200_mlp_dump(harm_ctx* c, const double* d_P, int stride, int phase, size_t max, float* d_feat,
                                  float* d_targ, int32_t* d_cell, size_t* n_out) {
  if (!c || !d_P || !d_feat || !d_targ || !n_out) return hb_setmsg("null argument", 1);
  if (stride < 1 || phase < 0 || phase >= stride) return hb_setmsg("need stride >= 1 and 0 <= phase < stride", 2);
  if (max > 0xFFFFFFF0ull) return hb_setmsg("max above 2^32-16 pairs", 2);
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  const long long ncell = (long long)d.n1 * d.n2 * d.n3;
  const long long nsel = (ncell - phase + stride - 1) / stride;
  unsigned int* cnt = c->d_nrare;  // free between substeps
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned int), c->stream));
  if (nsel > 0) {
    k_mlp_dump<<<nblk(nsel), 256, 0, c->stream>>>(d, ph, c->d_U, d_P, c->d_geom, stride, phase, (unsigned int)max,
                                                   d_feat, d_targ, d_cell, cnt);
    c->launches++;
    CK(cudaGetLastError());
  }
  unsigned int h = 0;
  CK(cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *n_out = (size_t)std::min<unsigned long long>(h, max);
  return 0;
}

extern "C" int harm_b200_mlp_synth(harm_ctx* c, size_t n, uint64_t seed, float* d_feat, float* d_targ, double* d_U,
                                   double* d_P, int32_t* d_cell) {
  if (!c || !d_feat || !d_targ) return hb_setmsg("null argument", 1);
  if (n == 0) return 0;
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  k_mlp_synth<<<nblk((long long)n), 256, 0, c->stream>>>(d, ph, n, seed, c->d_geom, c->d_aux, d_feat, d_targ, d_U, d_P,
                                                         d_cell);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}
