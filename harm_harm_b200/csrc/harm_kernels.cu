// harm_kernels.cu -- device kernels of the GRMHD step and the C ABI of libharm_b200.so.
//
// Kernels per RK substep (advance(), advance.c:140):
//   k_flux<DIR,T>   one thread per face: reconstruction of the primitives, B^dir
//                   continuity and limit_gamma at the face, L/R states and fluxes, vchar,
//                   HLL flux, CFL min (fluxcalc_standard flux.c:852, flux_compute_general
//                   fluxcompute.c:19).  The CFL minimum is a warp-shuffle/block reduction
//                   with one atomicMin per block on the IEEE bits of the positive dt.
//   k_emf<T>        one thread per cell corner: Toth corner EMFs from the field fluxes
//                   (flux_ct fluxct.c:186, CORNGDETVERSION=1).
//   k_update<T>     one thread per active cell: U_i = primtoU(p_i), flux divergence
//                   (flux2dUavg advance.c:1866) with the field fluxes rebuilt from the
//                   EMFs (fluxct.c:1110-1160), connection source of p_b (source_conn
//                   phys.c:132), RK combination (dUtoU advance.c:2046), FP64 Newton
//                   inversion with p_b as guess (Utoprimgen utoprimgen.c:32) and
//                   fixup1zone (fixup.c:561).
//   k_bound_x*      ghost zones (bound_prim step_ch.c:1332).
//   k_fixup_*       fixup_utoprim (fixup.c:1061) neighbour averaging, order independent.
//   k_finalize_dt   prepare_globaldt (advance.c:1558) and post_stepch (step_ch.c:213) on
//                   the device, so a run of steps never synchronises with the host.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include "harm_b200.h"
#include "harm_device.cuh"
#include "harm_invert.cuh"
#include "harm_ctx.cuh"

using namespace hb;

static __thread char g_errbuf[512];

static int seterr(const char* what, cudaError_t e) {
  snprintf(g_errbuf, sizeof(g_errbuf), "%s: %s", what, cudaGetErrorString(e));
  return 1;
}
#define CK(call)                                   \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return seterr(#call, e_); \
  } while (0)

extern "C" const char* harm_b200_last_error(void) { return g_errbuf; }

// ------------------------------------------------------------------ indexing helpers

struct Dims {
  int n1, n2, n3, ng, ng3, n1e, n2e, n3e;
  size_t plane, cells;
};

static Dims dims_of(const harm_grid& g) {
  Dims d;
  d.n1 = g.n1; d.n2 = g.n2; d.n3 = g.n3; d.ng = g.ng; d.ng3 = g.ng3;
  d.n1e = g.n1e; d.n2e = g.n2e; d.n3e = g.n3e;
  d.plane = (size_t)g.n1e * g.n2e;
  d.cells = d.plane * g.n3e;
  return d;
}

__device__ __forceinline__ size_t cidx(const Dims& d, int ii, int jj, int kk) {
  return ((size_t)kk * d.n2e + jj) * d.n1e + ii;
}

struct Phys {
  double gam, cour, gammamax, gammafail, defcon, safe;
  double dx1, dx2, dx3;
};

static Phys phys_of(const harm_grid& g) {
  Phys p;
  p.gam = g.gam; p.cour = g.cour; p.gammamax = g.gammamax; p.gammafail = g.gammafail;
  p.defcon = g.defcon; p.safe = g.safe;
  p.dx1 = g.dx[1]; p.dx2 = g.dx[2]; p.dx3 = g.dx[3];
  return p;
}

__device__ __forceinline__ unsigned long long dbl_bits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}

// block-wide min of a positive double, then one atomicMin on its bits
__device__ __forceinline__ void block_min_atomic(double v, unsigned long long* slot) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    int nw = (blockDim.x + 31) >> 5;
    v = (lane < nw) ? red[lane] : 1.e300;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0 && v < 1.e300) atomicMin(slot, dbl_bits(v));
  }
}

__device__ __forceinline__ void warp_add_atomic(double v, double* slot) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(slot, v);
}

// ------------------------------------------------------------------ flux kernel

// Face box of direction DIR (active-relative, inclusive): faces bounding active cells in
// DIR, one transverse ghost layer on each side of every other direction with n>1.
struct FaceBox {
  int lo[3], hi[3], cnt[3];
  long long n;
};

static FaceBox face_box(const Dims& d, int dir) {
  FaceBox b;
  int n[3] = {d.n1, d.n2, d.n3};
  for (int k = 0; k < 3; k++) {
    if (k == dir - 1) { b.lo[k] = 0; b.hi[k] = n[k]; }
    else if (n[k] > 1) { b.lo[k] = -1; b.hi[k] = n[k]; }
    else { b.lo[k] = 0; b.hi[k] = 0; }
    b.cnt[k] = b.hi[k] - b.lo[k] + 1;
  }
  b.n = (long long)b.cnt[0] * b.cnt[1] * b.cnt[2];
  return b;
}

template <typename T>
__device__ __forceinline__ void recon_face_mc(const double* __restrict__ P, size_t cells, size_t c0, long long stride,
                                              T* pl, T* pr) {
#pragma unroll
  for (int p = 0; p < NPR; p++) {
    const double* base = P + (size_t)p * cells + c0;
    T ym2 = (T)__ldg(base - 2 * stride), ym1 = (T)__ldg(base - stride), y0 = (T)__ldg(base), yp1 = (T)__ldg(base + stride);
    T dqm = mc_slope(ym2, ym1, y0), dq0 = mc_slope(ym1, y0, yp1);
    pl[p] = ym1 + T(0.5) * dqm;
    pr[p] = y0 - T(0.5) * dq0;
  }
}

template <int DIR, typename T, typename GT>
__global__ void __launch_bounds__(256) k_flux(Dims d, Phys ph, FaceBox fb, const double* __restrict__ P,
                                              const GT* __restrict__ geom, T* __restrict__ F,
                                              unsigned long long* __restrict__ dtslot) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double dtij = 1.e300;
  if (t < fb.n) {
    int a = (int)(t % fb.cnt[0]);
    long long r = t / fb.cnt[0];
    int b = (int)(r % fb.cnt[1]);
    int c = (int)(r / fb.cnt[1]);
    int ii = a + fb.lo[0] + d.ng, jj = b + fb.lo[1] + d.ng, kk = c + fb.lo[2] + d.ng3;
    size_t id = cidx(d, ii, jj, kk);
    long long stride = (DIR == 1) ? 1 : (DIR == 2) ? (long long)d.n1e : (long long)d.plane;
    T pl[NPR], pr[NPR];
    recon_face_mc<T>(P, d.cells, id, stride, pl, pr);
    constexpr int loc = (DIR == 1) ? HARM_LOC_FACE1 : (DIR == 2) ? HARM_LOC_FACE2 : HARM_LOC_CENT;
    Geo<T> g;
    load_geo<T, GT>(geom + (size_t)loc * HARM_NGF * d.plane, d.plane, (size_t)jj * d.n1e + ii, g);
    const int bp = HARM_B1 + DIR - 1;
    pl[bp] = pr[bp] = T(0.5) * (pl[bp] + pr[bp]);
    const T gam = (T)ph.gam, gmax = (T)ph.gammamax;
    limit_gamma<T>(gmax, pl, g);
    limit_gamma<T>(gmax, pr, g);
    State<T> ql, qr;
    get_state<T>(pl, g, gam, ql);
    get_state<T>(pr, g, gam, qr);
    T Fl[NPR], Fr[NPR], Ul[NPR], Ur[NPR];
    primtoflux<T>(pl, ql, DIR, g, g.gdet, Fl);
    primtoflux<T>(pl, ql, 0, g, g.gdet, Ul);
    primtoflux<T>(pr, qr, DIR, g, g.gdet, Fr);
    primtoflux<T>(pr, qr, 0, g, g.gdet, Ur);
    T cmaxl, cminl, cmaxr, cminr;
    vchar<T>(pl, ql, DIR, g, gam, cmaxl, cminl);
    vchar<T>(pr, qr, DIR, g, gam, cmaxr, cminr);
    T lmin = fmin(cminl, cminr), lmax = fmax(cmaxl, cmaxr);
    lmin = fabs(fmax(T(0), -lmin));
    lmax = fabs(fmax(T(0), lmax));
    const T cmin = lmin, cmax = lmax, ctop = fmax(lmax, lmin);
    if (cmax + cmin != T(0)) {
      const T inv = cmax + cmin;
#pragma unroll
      for (int p = 0; p < NPR; p++) F[(size_t)p * d.cells + id] = ((cmax * Fl[p] + cmin * Fr[p]) - (cmax * cmin) * (Ur[p] - Ul[p])) / inv;
    } else {
#pragma unroll
      for (int p = 0; p < NPR; p++) F[(size_t)p * d.cells + id] = T(0.5) * ((Fl[p] + Fr[p]) - ctop * (Ur[p] - Ul[p]));
    }
    const double dxd = (DIR == 1) ? ph.dx1 : (DIR == 2) ? ph.dx2 : ph.dx3;
    dtij = ph.cour * dxd / (double)ctop;
    if (!(dtij > 0.0)) dtij = 1.e300;
  }
  block_min_atomic(dtij, dtslot);
}

// ------------------------------------------------------------------ EMF kernel

template <typename T, typename GT>
__global__ void __launch_bounds__(256) k_emf(Dims d, const T* __restrict__ F1, const T* __restrict__ F2,
                                             const T* __restrict__ F3, const GT* __restrict__ geom, T* __restrict__ emf) {
  const int has3 = d.n3 > 1;
  const int c1n = d.n1 + 1, c2n = d.n2 + 1, c3n = has3 ? d.n3 + 1 : 1;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)c1n * c2n * c3n) return;
  int i = (int)(t % c1n);
  long long r = t / c1n;
  int j = (int)(r % c2n), k = (int)(r / c2n);
  int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
  int km = has3 ? kk - 1 : kk;
  const size_t cells = d.cells, plane = d.plane;
  auto ig = [&](int loc, int a, int b) -> T {
    return (T)__ldg(geom + ((size_t)loc * HARM_NGF + HARM_G_IGDET) * plane + (size_t)b * d.n1e + a);
  };
  auto gd = [&](int loc, int a, int b) -> T {
    return (T)__ldg(geom + ((size_t)loc * HARM_NGF + HARM_G_GDET) * plane + (size_t)b * d.n1e + a);
  };
  auto FF = [&](const T* Fa, int pl, int a, int b, int c) -> T { return Fa[(size_t)pl * cells + cidx(d, a, b, c)]; };
  T f2b3 = FF(F2, HARM_B3, ii, jj, kk) * ig(HARM_LOC_FACE2, ii, jj);
  T f2b3m = FF(F2, HARM_B3, ii, jj, km) * ig(HARM_LOC_FACE2, ii, jj);
  T f1b3 = FF(F1, HARM_B3, ii, jj, kk) * ig(HARM_LOC_FACE1, ii, jj);
  T f1b3m = FF(F1, HARM_B3, ii, jj, km) * ig(HARM_LOC_FACE1, ii, jj);
  T f1b2 = FF(F1, HARM_B2, ii, jj, kk) * ig(HARM_LOC_FACE1, ii, jj);
  T f1b2m = FF(F1, HARM_B2, ii, jj - 1, kk) * ig(HARM_LOC_FACE1, ii, jj - 1);
  T f2b1 = FF(F2, HARM_B1, ii, jj, kk) * ig(HARM_LOC_FACE2, ii, jj);
  T f2b1m = FF(F2, HARM_B1, ii - 1, jj, kk) * ig(HARM_LOC_FACE2, ii - 1, jj);
  T e1, e2, e3;
  if (has3) {
    T f3b2 = FF(F3, HARM_B2, ii, jj, kk) * ig(HARM_LOC_CENT, ii, jj);
    T f3b2m = FF(F3, HARM_B2, ii, jj - 1, kk) * ig(HARM_LOC_CENT, ii, jj - 1);
    T f3b1 = FF(F3, HARM_B1, ii, jj, kk) * ig(HARM_LOC_CENT, ii, jj);
    T f3b1m = FF(F3, HARM_B1, ii - 1, jj, kk) * ig(HARM_LOC_CENT, ii - 1, jj);
    e1 = T(0.25) * (+f2b3 + f2b3m - f3b2 - f3b2m);
    e2 = T(0.25) * (+f3b1 + f3b1m - f1b3 - f1b3m);
  } else {
    e1 = T(0.5) * (+f2b3 + f2b3m);
    e2 = T(0.5) * (-f1b3 - f1b3m);
  }
  e3 = T(0.25) * (+f1b2 + f1b2m - f2b1 - f2b1m);
  size_t id = cidx(d, ii, jj, kk);
  emf[id] = e1 * gd(HARM_LOC_FACE2, ii, jj);
  emf[cells + id] = e2 * gd(HARM_LOC_FACE1, ii, jj);
  emf[2 * cells + id] = e3 * gd(HARM_LOC_CORN3, ii, jj);
}

// ------------------------------------------------------------------ update + inversion

struct StepCoef {
  double CUf0, CUf2, Cun0, Cun1, Cun2;
  int finalstep;
  int guess;
};

template <typename T>
__device__ __forceinline__ double dU_cell(const Dims& d, int ii, int jj, int kk, int p, const T* __restrict__ F1,
                                          const T* __restrict__ F2, const T* __restrict__ F3, const T* __restrict__ emf,
                                          double idx1, double idx2, double idx3) {
  const size_t cells = d.cells;
  const int has3 = d.n3 > 1;
  const size_t id = cidx(d, ii, jj, kk);
  const size_t ip = cidx(d, ii + 1, jj, kk), jp = cidx(d, ii, jj + 1, kk), kp = has3 ? cidx(d, ii, jj, kk + 1) : id;
  double f1a, f1b, f2a, f2b, f3a = 0.0, f3b = 0.0;
  if (p < HARM_B1) {
    f1a = (double)F1[(size_t)p * cells + id]; f1b = (double)F1[(size_t)p * cells + ip];
    f2a = (double)F2[(size_t)p * cells + id]; f2b = (double)F2[(size_t)p * cells + jp];
    if (has3) { f3a = (double)F3[(size_t)p * cells + id]; f3b = (double)F3[(size_t)p * cells + kp]; }
  } else {
    const T* e1 = emf;
    const T* e2 = emf + cells;
    const T* e3 = emf + 2 * cells;
    auto E = [&](const T* e, int a, int b, int c) -> T { return e[cidx(d, a, b, c)]; };
    const int kq = has3 ? kk + 1 : kk;
    if (p == HARM_B1) {
      f1a = 0.0; f1b = 0.0;
      f2a = (double)(T(-0.5) * (E(e3, ii, jj, kk) + E(e3, ii + 1, jj, kk)));
      f2b = (double)(T(-0.5) * (E(e3, ii, jj + 1, kk) + E(e3, ii + 1, jj + 1, kk)));
      if (has3) {
        f3a = (double)(T(0.5) * (E(e2, ii, jj, kk) + E(e2, ii + 1, jj, kk)));
        f3b = (double)(T(0.5) * (E(e2, ii, jj, kk + 1) + E(e2, ii + 1, jj, kk + 1)));
      }
    } else if (p == HARM_B2) {
      f1a = (double)(T(0.5) * (E(e3, ii, jj, kk) + E(e3, ii, jj + 1, kk)));
      f1b = (double)(T(0.5) * (E(e3, ii + 1, jj, kk) + E(e3, ii + 1, jj + 1, kk)));
      f2a = 0.0; f2b = 0.0;
      if (has3) {
        f3a = (double)(T(-0.5) * (E(e1, ii, jj, kk) + E(e1, ii, jj + 1, kk)));
        f3b = (double)(T(-0.5) * (E(e1, ii, jj, kk + 1) + E(e1, ii, jj + 1, kk + 1)));
      }
    } else {
      f1a = (double)(T(-0.5) * (E(e2, ii, jj, kk) + E(e2, ii, jj, kq)));
      f1b = (double)(T(-0.5) * (E(e2, ii + 1, jj, kk) + E(e2, ii + 1, jj, kq)));
      f2a = (double)(T(0.5) * (E(e1, ii, jj, kk) + E(e1, ii, jj, kq)));
      f2b = (double)(T(0.5) * (E(e1, ii, jj + 1, kk) + E(e1, ii, jj + 1, kq)));
      f3a = 0.0; f3b = 0.0;
    }
  }
  double d1 = -(f1b - f1a) * idx1;
  double d2 = -(f2b - f2a) * idx2;
  double d3 = has3 ? -(f3b - f3a) * idx3 : 0.0;
  return d1 + d2 + d3;
}

// connection source (source_conn): dU^{UU+l} = gdet [ T^j_k Gamma^k_{l j} - rho u^j Gamma^t_{l j} ]
__device__ __forceinline__ void source_conn(const double* pr, const State<double>& q, const Geo<double>& g,
                                            const double* __restrict__ conn, size_t plane, size_t c2, double* dUg) {
  double mhd[4][4];
#pragma unroll
  for (int j = 0; j < 4; j++) {
    double F[NPR];
    primtoflux<double>(pr, q, j, g, 1.0, F);
#pragma unroll
    for (int k = 0; k < 4; k++) mhd[j][k] = F[HARM_UU + k];
  }
#pragma unroll
  for (int l = 0; l < 4; l++) {
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int k = 0; k < 4; k++) s += mhd[j][k] * __ldg(conn + (size_t)((k * 4 + l) * 4 + j) * plane + c2);
#pragma unroll
    for (int j = 0; j < 4; j++) s += -pr[HARM_RHO] * q.ucon[j] * __ldg(conn + (size_t)((0 * 4 + l) * 4 + j) * plane + c2);
    dUg[HARM_UU + l] = g.gdet * s;
  }
  dUg[HARM_RHO] = g.gdet * 0.0;
  dUg[HARM_B1] = g.gdet * 0.0;
  dUg[HARM_B2] = g.gdet * 0.0;
  dUg[HARM_B3] = g.gdet * 0.0;
}

// fixup1zone with FIXUPTYPE 1; returns floor-hit indicator, updates pr/flag/iters
__device__ __forceinline__ int fixup1zone(double* pr, const Geo<double>& g, double rhofl, double ufl, double gam,
                                          double gammamax, double gammafail, int8_t& flag, int& iters) {
  double prnew[NPR];
  int did = 0;
  rhofl = (rhofl < kSMALL) ? kSMALL : rhofl;
  ufl = (ufl < kSMALL) ? kSMALL : ufl;
#pragma unroll
  for (int pl = 0; pl < NPR; pl++) prnew[pl] = pr[pl];
  if (rhofl > pr[HARM_RHO]) { did = 1; prnew[HARM_RHO] = rhofl; }
  if (ufl > pr[HARM_UU]) { did = 1; prnew[HARM_UU] = ufl; }
  if (did) {
    State<double> q, dq;
    double U[NPR], dU[NPR], dpr[NPR];
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) dpr[pl] = 0.0;
    get_state<double>(pr, g, gam, q);
    primtoflux<double>(pr, q, 0, g, 1.0, U);
    dpr[HARM_RHO] = prnew[HARM_RHO] - pr[HARM_RHO];
    dpr[HARM_UU] = prnew[HARM_UU] - pr[HARM_UU];
    get_state<double>(dpr, g, gam, dq);
    primtoflux<double>(dpr, dq, 0, g, 1.0, dU);
#pragma unroll
    for (int pl = 0; pl < NPR; pl++) U[pl] += dU[pl];
    iters += utoprimgen(U, g, 1.0, pr, flag, gam, gammafail, false, 0.0, nullptr);
    if (flag > 0) {
#pragma unroll
      for (int pl = 0; pl < NPR; pl++) pr[pl] = prnew[pl];
    }
  }
  limit_gamma<double>(gammamax, pr, g);
  return did;
}

template <typename T>
__global__ void __launch_bounds__(256) k_update(Dims d, Phys ph, StepCoef sc, const double* __restrict__ dtp,
                                                const double* pi, const double* pb, double* pf,
                                                int8_t* __restrict__ pflag, const T* __restrict__ F1,
                                                const T* __restrict__ F2, const T* __restrict__ F3,
                                                const T* __restrict__ emf, const double* __restrict__ geom,
                                                const double* __restrict__ conn, const double* __restrict__ aux,
                                                const float* __restrict__ mlp, double* __restrict__ stats) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long ncell = (long long)d.n1 * d.n2 * d.n3;
  double iters_d = 0.0, fails = 0.0, floors = 0.0, fallbacks = 0.0;
  if (t < ncell) {
    int i = (int)(t % d.n1);
    long long r = t / d.n1;
    int j = (int)(r % d.n2), k = (int)(r / d.n2);
    int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
    const size_t id = cidx(d, ii, jj, kk), c2 = (size_t)jj * d.n1e + ii;
    Geo<double> g;
    load_geo<double, double>(geom, d.plane, c2, g);
    double pri[NPR], prb[NPR];
#pragma unroll
    for (int p = 0; p < NPR; p++) { pri[p] = pi[(size_t)p * d.cells + id]; prb[p] = pb[(size_t)p * d.cells + id]; }
    State<double> qi, qb;
    get_state<double>(pri, g, ph.gam, qi);
    double Ui[NPR];
    primtoflux<double>(pri, qi, 0, g, g.gdet, Ui);
    const double idx1 = 1.0 / ph.dx1, idx2 = 1.0 / ph.dx2, idx3 = 1.0 / ph.dx3;
    get_state<double>(prb, g, ph.gam, qb);
    double dUg[NPR];
    source_conn(prb, qb, g, conn, d.plane, c2, dUg);
    const double dt = *dtp;
    double U[NPR];
#pragma unroll
    for (int p = 0; p < NPR; p++) {
      double dU = dU_cell<T>(d, ii, jj, kk, p, F1, F2, F3, emf, idx1, idx2, idx3);
      double Uf = sc.CUf0 * Ui[p] + sc.CUf2 * dt * (dU + dUg[p]);
      double ucum = sc.Cun0 * Ui[p] + sc.Cun1 * dt * (dU + dUg[p]) + sc.Cun2 * Uf;
      U[p] = sc.finalstep ? ucum : Uf;
    }
    int8_t flag = 0;
    double pr[NPR];
#pragma unroll
    for (int p = 0; p < NPR; p++) pr[p] = prb[p];
    bool gfail = false;
    int it = utoprimgen(U, g, g.igdet, pr, flag, ph.gam, ph.gammafail, false, 0.0, &gfail);
    if (gfail) fallbacks = 1.0;
    if (flag > 0) fails = 1.0;
    floors = (double)fixup1zone(pr, g, __ldg(aux + (size_t)HARM_AUX_RHOFLOOR * d.plane + c2),
                                __ldg(aux + (size_t)HARM_AUX_UFLOOR * d.plane + c2), ph.gam, ph.gammamax, ph.gammafail,
                                flag, it);
    iters_d = (double)it;
    pflag[id] = flag;
#pragma unroll
    for (int p = 0; p < NPR; p++) pf[(size_t)p * d.cells + id] = pr[p];
  }
  if (stats) {
    warp_add_atomic(iters_d, stats + 0);
    warp_add_atomic(fails, stats + 3);
    warp_add_atomic(floors, stats + 4);
    warp_add_atomic(fallbacks, stats + 2);
  }
}

// copy p_b into the ghost zones of p_f (advance.c:654 copies the full grid)
__global__ void k_copy_ghosts(Dims d, const double* __restrict__ pb, double* __restrict__ pf) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)d.cells) return;
  int ii = (int)(t % d.n1e);
  long long r = t / d.n1e;
  int jj = (int)(r % d.n2e), kk = (int)(r / d.n2e);
  bool active = ii >= d.ng && ii < d.ng + d.n1 && jj >= d.ng && jj < d.ng + d.n2 && kk >= d.ng3 && kk < d.ng3 + d.n3;
  if (active) return;
#pragma unroll
  for (int p = 0; p < NPR; p++) pf[(size_t)p * d.cells + t] = pb[(size_t)p * d.cells + t];
}

// ------------------------------------------------------------------ boundary conditions

__global__ void k_bound_x1(Dims d, Phys ph, double* P, int8_t* flag, const double* __restrict__ geom) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)2 * d.ng * d.n2e * d.n3e;
  if (t >= n) return;
  int gq = (int)(t % (2 * d.ng));
  long long r = t / (2 * d.ng);
  int jj = (int)(r % d.n2e), kk = (int)(r / d.n2e);
  if (gq < d.ng) {
    int ii = gq;
    size_t dst = cidx(d, ii, jj, kk), src = cidx(d, d.ng, jj, kk);
    if (P)
      for (int p = 0; p < NPR; p++) P[(size_t)p * d.cells + dst] = P[(size_t)p * d.cells + src];
    if (flag) flag[dst] = flag[src];
  } else {
    int ii = d.ng + d.n1 + (gq - d.ng);
    size_t dst = cidx(d, ii, jj, kk), src = cidx(d, d.ng + d.n1 - 1, jj, kk);
    if (flag) flag[dst] = flag[src];
    if (!P) return;
    double pr[NPR];
    for (int p = 0; p < NPR; p++) pr[p] = P[(size_t)p * d.cells + src];
    Geo<double> g;
    load_geo<double, double>(geom, d.plane, (size_t)jj * d.n1e + ii, g);
    // inflow_check_rel4vel (fixup.c:3255) for the outer radial boundary
    double ucon[4], gamma, qsq;
    ucon_of<double>(pr, g, ucon, gamma, qsq);
    if (ucon[1] < 0.) {
      pr[HARM_U1] /= gamma; pr[HARM_U2] /= gamma; pr[HARM_U3] /= gamma;
      double alpha = 1. / sqrt(-g.gcon[0]);
      double betacon = g.gcon[1] * alpha * alpha;
      pr[HARM_U1] = betacon / alpha;
      double vsq = 0.;
      for (int a = 1; a < 4; a++)
        for (int b = 1; b < 4; b++) vsq += g.gcov[sym(a, b)] * pr[HARM_U1 + a - 1] * pr[HARM_U1 + b - 1];
      if (vsq < 0.0 && vsq > -2.220446049250313e-16 * 100.0) vsq = 0.0;
      if (vsq >= 1.0) vsq = 1.0 - 1.0 / (ph.gammamax * ph.gammamax);
      gamma = 1. / sqrt(1. - vsq);
      pr[HARM_U1] *= gamma; pr[HARM_U2] *= gamma; pr[HARM_U3] *= gamma;
    }
    limit_gamma<double>(ph.gammamax, pr, g);
    for (int p = 0; p < NPR; p++) P[(size_t)p * d.cells + dst] = pr[p];
  }
}

__global__ void k_bound_x2(Dims d, double* P, int8_t* flag) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)2 * d.ng * d.n1e * d.n3e;
  if (t >= n) return;
  int ii = (int)(t % d.n1e);
  long long r = t / d.n1e;
  int gq = (int)(r % (2 * d.ng)), kk = (int)(r / (2 * d.ng));
  int k = kk - d.ng3;
  int ks = (d.n3 > 1) ? ((k + d.n3 / 2) % d.n3 + d.n3) % d.n3 + d.ng3 : kk;
  int jj, js;
  if (gq < d.ng) { jj = gq; js = 2 * d.ng - 1 - jj; }
  else { jj = d.ng + d.n2 + (gq - d.ng); js = 2 * (d.ng + d.n2) - 1 - jj; }
  size_t dst = cidx(d, ii, jj, kk), src = cidx(d, ii, js, ks);
  if (flag) flag[dst] = flag[src];
  if (!P) return;
  for (int p = 0; p < NPR; p++) {
    double v = P[(size_t)p * d.cells + src];
    if (p == HARM_U2 || p == HARM_B2) v = -v;
    P[(size_t)p * d.cells + dst] = v;
  }
}

__global__ void k_bound_x3(Dims d, double* P, int8_t* flag) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)2 * d.ng3 * d.plane;
  if (t >= n) return;
  int ii = (int)(t % d.n1e);
  long long r = t / d.n1e;
  int jj = (int)(r % d.n2e), gq = (int)(r / d.n2e);
  int kk, ks;
  if (gq < d.ng3) { kk = gq; ks = kk + d.n3; }
  else { kk = d.ng3 + d.n3 + (gq - d.ng3); ks = kk - d.n3; }
  size_t dst = cidx(d, ii, jj, kk), src = cidx(d, ii, jj, ks);
  if (flag) flag[dst] = flag[src];
  if (P)
    for (int p = 0; p < NPR; p++) P[(size_t)p * d.cells + dst] = P[(size_t)p * d.cells + src];
}

// ------------------------------------------------------------------ post_fixup

struct FixRec {
  long long id;
  double v[5];
};

__global__ void __launch_bounds__(256) k_fixup_compute(Dims d, Phys ph, const double* __restrict__ P,
                                                       const int8_t* __restrict__ flag, const double* __restrict__ geom,
                                                       FixRec* __restrict__ recs, unsigned int* __restrict__ nrec,
                                                       unsigned int cap) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)d.n1 * d.n2 * d.n3) return;
  int i = (int)(t % d.n1);
  long long r = t / d.n1;
  int j = (int)(r % d.n2), k = (int)(r / d.n2);
  int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
  size_t id = cidx(d, ii, jj, kk);
  int8_t f = flag[id];
  if (f <= 0) return;
  int startpl, endpl;
  const bool u2 = (f == HARM_UTOPRIMFAILU2AVG1 || f == HARM_UTOPRIMFAILU2AVG2);
  if (u2 || f == 13) { startpl = endpl = HARM_UU; }
  else { startpl = HARM_RHO; endpl = HARM_U3; }
  const int s1 = d.n1 > 1, s2 = d.n2 > 1, s3 = d.n3 > 1;
  const int rnx = s1 ? 3 : 1, rny = s2 ? 3 : 1;
  const int npairs = ((s1 + s2 + s3) == 3 ? 27 : (s1 + s2 + s3) == 2 ? 9 : 3) / 2;
  double sum0[5] = {0, 0, 0, 0, 0}, sum1[5] = {0, 0, 0, 0, 0}, lastmin[5];
  for (int p = 0; p < 5; p++) lastmin[p] = 1E50;
  int numavg0 = 0, numavg1 = 0;
  const double ref = P[(size_t)HARM_UU * d.cells + id];
  for (int qq = 0; qq < npairs; qq++) {
    int di = (qq % rnx) - s1, dj = ((qq % (rnx * rny)) / rnx) - s2, dk = (qq / (rnx * rny)) - s3;
    size_t a = cidx(d, ii + di, jj + dj, kk + dk), b = cidx(d, ii - di, jj - dj, kk - dk);
    int thisok = flag[a] <= 0, thatok = flag[b] <= 0;
    numavg0 += thisok + thatok;
    for (int p = startpl; p <= endpl; p++) {
      double fa = P[(size_t)p * d.cells + a], fb = P[(size_t)p * d.cells + b];
      if (!u2) {
        double add = fa * thisok + fb * thatok;
        if (qq % 2 == 0) sum0[p] += add; else sum1[p] += add;
      } else if (fa >= ref && fb >= ref) {
        lastmin[p] = fmin(fmin(lastmin[p], fa), fb);
        numavg1++;
      }
    }
  }
  double out[5];
  for (int p = 0; p < 5; p++) out[p] = P[(size_t)p * d.cells + id];
  if (!u2) {
    if (numavg0 != 0)
      for (int p = startpl; p <= endpl; p++) out[p] = (sum0[p] + sum1[p]) / (double)numavg0;
  } else {
    if (numavg1 != 0)
      for (int p = startpl; p <= endpl; p++) out[p] = lastmin[p];
  }
  if (startpl <= HARM_U1 && endpl >= HARM_U3) {
    Geo<double> g;
    load_geo<double, double>(geom, d.plane, (size_t)jj * d.n1e + ii, g);
    double pa[NPR], pv[NPR];
    for (int p = 0; p < NPR; p++) pa[p] = P[(size_t)p * d.cells + id];
    for (int p = 0; p < NPR; p++) pv[p] = (p < 5) ? out[p] : pa[p];
    double ucon[4], gamma, qsq;
    ucon_of<double>(pa, g, ucon, gamma, qsq);
    if (gamma > ph.gammamax) gamma = ph.gammamax;
    limit_gamma<double>(gamma, pv, g);
    for (int p = 0; p < 5; p++) out[p] = pv[p];
  }
  unsigned int slot = atomicAdd(nrec, 1u);
  if (slot < cap) {
    recs[slot].id = (long long)id;
    for (int p = 0; p < 5; p++) recs[slot].v[p] = out[p];
  }
}

__global__ void k_fixup_apply(Dims d, double* __restrict__ P, const FixRec* __restrict__ recs,
                              const unsigned int* __restrict__ nrec, unsigned int cap) {
  unsigned int n = *nrec;
  if (n > cap) n = cap;
  for (unsigned int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    size_t id = (size_t)recs[s].id;
    for (int p = 0; p < 5; p++) P[(size_t)p * d.cells + id] = recs[s].v[p];
  }
}

// ------------------------------------------------------------------ dt

// slots[6]: per substep s (0,1) and direction d the atomic min of cour dx/ctop.
__global__ void k_finalize_dt(Phys ph, unsigned long long* slots, double* dt, double* ndt_out, int nsub) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double last = 1.e100;
  for (int s = 0; s < nsub; s++) {
    double nd[3];
    for (int q = 0; q < 3; q++) {
      unsigned long long b = slots[s * 3 + q];
      nd[q] = (b == 0xFFFFFFFFFFFFFFFFull) ? 1.e100 : __longlong_as_double((long long)b);
    }
    double wavedt = 1. / (1. / nd[0] + 1. / nd[1] + 1. / nd[2]);
    double ndt = ph.defcon * fmin(wavedt, 1.e100);
    if (ndt_out) ndt_out[s] = ndt;
    if (ndt < last) last = ndt;
  }
  if (dt) {
    double cur = *dt;
    if (last > ph.safe * cur) last = ph.safe * cur;
    *dt = last;
  }
  for (int q = 0; q < 3 * nsub; q++) slots[q] = 0xFFFFFFFFFFFFFFFFull;
}

// ------------------------------------------------------------------ points inversion

__global__ void k_utoprim_points(size_t n, Phys ph, const double* __restrict__ U, const double* __restrict__ geom,
                                 double* __restrict__ P, int8_t* __restrict__ pflag, int32_t* __restrict__ iters) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  Geo<double> g;
  load_geo<double, double>(geom, n, t, g);
  double u[NPR], pr[NPR];
  for (int p = 0; p < NPR; p++) { u[p] = U[(size_t)p * n + t]; pr[p] = P[(size_t)p * n + t]; }
  int8_t flag = 0;
  int it = utoprimgen(u, g, g.igdet, pr, flag, ph.gam, ph.gammafail, false, 0.0, nullptr);
  for (int p = 0; p < NPR; p++) P[(size_t)p * n + t] = pr[p];
  pflag[t] = flag;
  if (iters) iters[t] = it;
}

// ------------------------------------------------------------------ host side

static inline unsigned int nblk(long long n, int bs = 256) { return (unsigned int)((n + bs - 1) / bs); }

extern "C" int harm_b200_create(const harm_grid* g, const double* geom_h, const double* conn_h, const double* aux_h,
                                int device, harm_ctx** out) {
  if (!g || !geom_h || !conn_h || !aux_h || !out) { snprintf(g_errbuf, sizeof(g_errbuf), "null argument"); return 1; }
  if (g->lim != HARM_LIM_MC) {
    snprintf(g_errbuf, sizeof(g_errbuf), "reconstruction %d not available in this build", g->lim);
    return 2;
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
  CK(cudaMemcpy(c->d_geom, geom_h, gsz * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_conn, conn_h, 64 * d.plane * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_aux, aux_h, HARM_NAUX * d.plane * sizeof(double), cudaMemcpyHostToDevice));
  {
    float* tmp = (float*)malloc(gsz * sizeof(float));
    for (size_t q = 0; q < gsz; q++) tmp[q] = (float)geom_h[q];
    CK(cudaMemcpy(c->d_geomf, tmp, gsz * sizeof(float), cudaMemcpyHostToDevice));
    free(tmp);
  }
  for (int q = 0; q < 3; q++) {
    CK(cudaMalloc(&c->d_F[q], NPR * d.cells * sizeof(double)));
    CK(cudaMalloc(&c->d_Ff[q], NPR * d.cells * sizeof(float)));
  }
  CK(cudaMalloc(&c->d_emf, 3 * d.cells * sizeof(double)));
  CK(cudaMalloc(&c->d_emff, 3 * d.cells * sizeof(float)));
  CK(cudaMalloc(&c->d_pk, NPR * d.cells * sizeof(double)));
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
  CK(cudaMemset(c->d_dtslots, 0xFF, 6 * sizeof(unsigned long long)));
  CK(cudaMallocHost(&c->h_scal, 64 * sizeof(double)));
  *out = c;
  return 0;
}

extern "C" int harm_b200_destroy(harm_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  void* ptrs[] = {c->d_geom, c->d_geomf, c->d_conn, c->d_aux, c->d_F[0], c->d_F[1], c->d_F[2], c->d_Ff[0], c->d_Ff[1],
                  c->d_Ff[2], c->d_emf, c->d_emff, c->d_pk, c->d_pflag, c->d_fixrec, c->d_scal, c->d_Pdev, c->d_mlp,
                  c->d_mlp_master, c->d_mlp_adam, c->d_mlp_work};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->h_scal) cudaFreeHost(c->h_scal);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return 0;
}

extern "C" void* harm_b200_stream(harm_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" unsigned long long harm_b200_launch_count(harm_ctx* c) { return c ? c->launches : 0ull; }

extern "C" int harm_b200_bound(harm_ctx* c, double* d_P) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  k_bound_x1<<<nblk(2LL * d.ng * d.n2e * d.n3e), 256, 0, c->stream>>>(d, ph, d_P, nullptr, c->d_geom);
  c->launches++;
  k_bound_x2<<<nblk(2LL * d.ng * d.n1e * d.n3e), 256, 0, c->stream>>>(d, d_P, nullptr);
  c->launches++;
  if (d.n3 > 1) { k_bound_x3<<<nblk(2LL * d.ng3 * (long long)d.plane), 256, 0, c->stream>>>(d, d_P, nullptr); c->launches++; }
  CK(cudaGetLastError());
  return 0;
}

static int bound_flags(harm_ctx* c, int8_t* flag) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  k_bound_x1<<<nblk(2LL * d.ng * d.n2e * d.n3e), 256, 0, c->stream>>>(d, ph, nullptr, flag, c->d_geom);
  c->launches++;
  k_bound_x2<<<nblk(2LL * d.ng * d.n1e * d.n3e), 256, 0, c->stream>>>(d, nullptr, flag);
  c->launches++;
  if (d.n3 > 1) { k_bound_x3<<<nblk(2LL * d.ng3 * (long long)d.plane), 256, 0, c->stream>>>(d, nullptr, flag); c->launches++; }
  CK(cudaGetLastError());
  return 0;
}

// launch the three flux kernels and the EMF kernel for p_b; dt minima into slots[3]
template <typename T>
static int launch_fluxes(harm_ctx* c, const double* d_pb, T* F1, T* F2, T* F3, T* emf, unsigned long long* slots) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  const bool fp32 = sizeof(T) == 4;
  FaceBox b1 = face_box(d, 1), b2 = face_box(d, 2), b3 = face_box(d, 3);
  if (fp32) {
    k_flux<1, T, float><<<nblk(b1.n), 256, 0, c->stream>>>(d, ph, b1, d_pb, c->d_geomf, F1, slots + 0);
    c->launches++;
    k_flux<2, T, float><<<nblk(b2.n), 256, 0, c->stream>>>(d, ph, b2, d_pb, c->d_geomf, F2, slots + 1);
    c->launches++;
    if (d.n3 > 1) { k_flux<3, T, float><<<nblk(b3.n), 256, 0, c->stream>>>(d, ph, b3, d_pb, c->d_geomf, F3, slots + 2); c->launches++; }
  } else {
    k_flux<1, T, double><<<nblk(b1.n), 256, 0, c->stream>>>(d, ph, b1, d_pb, c->d_geom, F1, slots + 0);
    c->launches++;
    k_flux<2, T, double><<<nblk(b2.n), 256, 0, c->stream>>>(d, ph, b2, d_pb, c->d_geom, F2, slots + 1);
    c->launches++;
    if (d.n3 > 1) { k_flux<3, T, double><<<nblk(b3.n), 256, 0, c->stream>>>(d, ph, b3, d_pb, c->d_geom, F3, slots + 2); c->launches++; }
  }
  long long nc = (long long)(d.n1 + 1) * (d.n2 + 1) * (d.n3 > 1 ? d.n3 + 1 : 1);
  if (fp32)
    k_emf<T, float><<<nblk(nc), 256, 0, c->stream>>>(d, F1, F2, F3, c->d_geomf, emf);
  else
    k_emf<T, double><<<nblk(nc), 256, 0, c->stream>>>(d, F1, F2, F3, c->d_geom, emf);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

// field fluxes of the faces of active cells from the EMFs (for the standalone fluxcalc)
template <typename T>
__global__ void k_emf_to_flux(Dims d, const T* __restrict__ emf, T* F1, T* F2, T* F3) {
  const int has3 = d.n3 > 1;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c1n = d.n1 + 1, c2n = d.n2 + 1, c3n = has3 ? d.n3 + 1 : 1;
  if (t >= (long long)c1n * c2n * c3n) return;
  int i = (int)(t % c1n);
  long long r = t / c1n;
  int j = (int)(r % c2n), k = (int)(r / c2n);
  int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
  const size_t cells = d.cells;
  auto E = [&](int q, int a, int b, int cc) -> T { return emf[(size_t)q * cells + cidx(d, a, b, cc)]; };
  size_t id = cidx(d, ii, jj, kk);
  int kp = has3 ? kk + 1 : kk;
  if (k < d.n3 && j < d.n2) {
    F1[(size_t)HARM_B1 * cells + id] = T(0);
    F1[(size_t)HARM_B2 * cells + id] = T(0.5) * (E(2, ii, jj, kk) + E(2, ii, jj + 1, kk));
    F1[(size_t)HARM_B3 * cells + id] = T(-0.5) * (E(1, ii, jj, kk) + E(1, ii, jj, kp));
  }
  if (k < d.n3 && i < d.n1) {
    F2[(size_t)HARM_B1 * cells + id] = T(-0.5) * (E(2, ii, jj, kk) + E(2, ii + 1, jj, kk));
    F2[(size_t)HARM_B2 * cells + id] = T(0);
    F2[(size_t)HARM_B3 * cells + id] = T(0.5) * (E(0, ii, jj, kk) + E(0, ii, jj, kp));
  }
  if (has3 && i < d.n1 && j < d.n2) {
    F3[(size_t)HARM_B1 * cells + id] = T(0.5) * (E(1, ii, jj, kk) + E(1, ii + 1, jj, kk));
    F3[(size_t)HARM_B2 * cells + id] = T(-0.5) * (E(0, ii, jj, kk) + E(0, ii, jj + 1, kk));
    F3[(size_t)HARM_B3 * cells + id] = T(0);
  }
}

extern "C" int harm_b200_fluxcalc(harm_ctx* c, int precision, const double* d_pb, double* d_F1, double* d_F2,
                                  double* d_F3, double ndt[3]) {
  if (precision != HARM_PREC_FP64) { snprintf(g_errbuf, sizeof(g_errbuf), "fluxcalc into FP64 arrays needs HARM_PREC_FP64"); return 2; }
  Dims d = dims_of(c->g);
  unsigned long long* slots = c->d_dtslots;
  CK(cudaMemsetAsync(slots, 0xFF, 3 * sizeof(unsigned long long), c->stream));
  if (launch_fluxes<double>(c, d_pb, d_F1, d_F2, d_F3, c->d_emf, slots)) return 1;
  long long nc = (long long)(d.n1 + 1) * (d.n2 + 1) * (d.n3 > 1 ? d.n3 + 1 : 1);
  k_emf_to_flux<double><<<nblk(nc), 256, 0, c->stream>>>(d, c->d_emf, d_F1, d_F2, d_F3);
  c->launches++;
  CK(cudaGetLastError());
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

// one substep on the device; dt from d_dt, dt minima of this substep into slots
static int substep(harm_ctx* c, int precision, int guess, int timeorder, int numtimeorders, const double* d_pi,
                   const double* d_pb, double* d_pf, int8_t* d_pflag, const double* CUf, const double* Cunew,
                   unsigned long long* slots, bool with_stats) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  StepCoef sc;
  sc.CUf0 = CUf[0]; sc.CUf2 = CUf[2];
  sc.Cun0 = Cunew[0]; sc.Cun1 = Cunew[1]; sc.Cun2 = Cunew[2];
  sc.finalstep = (timeorder == numtimeorders - 1);
  sc.guess = guess;
  long long ncell = (long long)d.n1 * d.n2 * d.n3;
  double* st = with_stats ? c->d_stats : nullptr;
  if (precision == HARM_PREC_FP64) {
    if (launch_fluxes<double>(c, d_pb, c->d_F[0], c->d_F[1], c->d_F[2], c->d_emf, slots)) return 1;
    k_update<double><<<nblk(ncell), 256, 0, c->stream>>>(d, ph, sc, c->d_dt, d_pi, d_pb, d_pf, d_pflag, c->d_F[0],
                                                         c->d_F[1], c->d_F[2], c->d_emf, c->d_geom, c->d_conn, c->d_aux,
                                                         c->d_mlp, st);
    c->launches++;
  } else {
    if (launch_fluxes<float>(c, d_pb, c->d_Ff[0], c->d_Ff[1], c->d_Ff[2], c->d_emff, slots)) return 1;
    k_update<float><<<nblk(ncell), 256, 0, c->stream>>>(d, ph, sc, c->d_dt, d_pi, d_pb, d_pf, d_pflag, c->d_Ff[0],
                                                        c->d_Ff[1], c->d_Ff[2], c->d_emff, c->d_geom, c->d_conn, c->d_aux,
                                                        c->d_mlp, st);
    c->launches++;
  }
  CK(cudaGetLastError());
  return 0;
}

extern "C" int harm_b200_advance(harm_ctx* c, int precision, int guess, int timeorder, int numtimeorders,
                                 const double* d_pi, const double* d_pb, double* d_pf, int8_t* d_pflag, double dt,
                                 const double CUf[4], const double Cunew[4], double* ndt, harm_stats* stats) {
  Dims d = dims_of(c->g);
  c->h_scal[0] = dt;
  CK(cudaMemcpyAsync(c->d_dt, c->h_scal, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->d_stats, 0, 5 * sizeof(double), c->stream));
  if (substep(c, precision, guess, timeorder, numtimeorders, d_pi, d_pb, d_pf, d_pflag, CUf, Cunew, c->d_dtslots, true))
    return 1;
  k_copy_ghosts<<<nblk((long long)d.cells), 256, 0, c->stream>>>(d, d_pb, d_pf);
  c->launches++;
  Phys ph = phys_of(c->g);
  k_finalize_dt<<<1, 32, 0, c->stream>>>(ph, c->d_dtslots, nullptr, c->d_ndt, 1);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->h_scal + 1, c->d_ndt, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->h_scal + 8, c->d_stats, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (ndt) *ndt = c->h_scal[1];
  if (stats) {
    stats->newton_iters += c->h_scal[8];
    stats->cells_inverted += (double)d.n1 * d.n2 * d.n3;
    stats->mlp_fallbacks += c->h_scal[10];
    stats->inversion_failures += c->h_scal[11];
    stats->floor_hits += c->h_scal[12];
  }
  return 0;
}

extern "C" int harm_b200_post_fixup(harm_ctx* c, double* d_pf, int8_t* d_pflag) {
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  if (bound_flags(c, d_pflag)) return 1;
  CK(cudaMemsetAsync(c->d_nrec, 0, sizeof(unsigned int), c->stream));
  long long ncell = (long long)d.n1 * d.n2 * d.n3;
  k_fixup_compute<<<nblk(ncell), 256, 0, c->stream>>>(d, ph, d_pf, d_pflag, c->d_geom, (FixRec*)c->d_fixrec, c->d_nrec,
                                                       c->fix_cap);
  c->launches++;
  k_fixup_apply<<<4 * 148, 256, 0, c->stream>>>(d, d_pf, (const FixRec*)c->d_fixrec, c->d_nrec, c->fix_cap);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

// enqueue one full RK2 step with dt in d_dt (no host synchronisation)
static int enqueue_step(harm_ctx* c, int precision, int guess, double* d_P, bool with_stats) {
  static const double CUf[2][4] = {{1.0, 0.0, 0.5, 0.0}, {1.0, 0.0, 1.0, 0.0}};
  static const double Cun[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 1.0, 0.5}};
  Phys ph = phys_of(c->g);
  if (substep(c, precision, guess, 0, 2, d_P, d_P, c->d_pk, c->d_pflag, CUf[0], Cun[0], c->d_dtslots, with_stats)) return 1;
  if (harm_b200_bound(c, c->d_pk)) return 1;
  if (harm_b200_post_fixup(c, c->d_pk, c->d_pflag)) return 1;
  if (harm_b200_bound(c, c->d_pk)) return 1;
  if (substep(c, precision, guess, 1, 2, d_P, c->d_pk, d_P, c->d_pflag, CUf[1], Cun[1], c->d_dtslots + 3, with_stats))
    return 1;
  if (harm_b200_bound(c, d_P)) return 1;
  if (harm_b200_post_fixup(c, d_P, c->d_pflag)) return 1;
  if (harm_b200_bound(c, d_P)) return 1;
  k_finalize_dt<<<1, 32, 0, c->stream>>>(ph, c->d_dtslots, c->d_dt, c->d_ndt, 2);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
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
  *dt = c->h_scal[0];
  if (stats) {
    stats->newton_iters += c->h_scal[8];
    stats->cells_inverted += 2.0 * nsteps * (double)d.n1 * d.n2 * d.n3;
    stats->mlp_fallbacks += c->h_scal[10];
    stats->inversion_failures += c->h_scal[11];
    stats->floor_hits += c->h_scal[12];
  }
  return 0;
}

extern "C" int harm_b200_step(harm_ctx* c, int precision, int guess, double* d_P, double* dt, harm_stats* stats) {
  return harm_b200_step_n(c, precision, guess, d_P, 1, dt, stats);
}

extern "C" int harm_b200_step_host(harm_ctx* c, int precision, int guess, double* h_P, double* dt, harm_stats* stats) {
  size_t bytes = NPR * c->cells * sizeof(double);
  if (!c->d_Pdev) CK(cudaMalloc(&c->d_Pdev, bytes));
  CK(cudaMemcpyAsync(c->d_Pdev, h_P, bytes, cudaMemcpyHostToDevice, c->stream));
  if (harm_b200_step_n(c, precision, guess, c->d_Pdev, 1, dt, stats)) return 1;
  CK(cudaMemcpyAsync(h_P, c->d_Pdev, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int harm_b200_utoprimgen_points(harm_ctx* c, size_t n, int guess, const double* d_U, const double* d_geom,
                                           double* d_P, int8_t* d_pflag, int32_t* d_iters) {
  (void)guess;
  if (n == 0) return 0;
  Phys ph = phys_of(c->g);
  k_utoprim_points<<<nblk((long long)n), 256, 0, c->stream>>>(n, ph, d_U, d_geom, d_P, d_pflag, d_iters);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// Time the stages of one substep (substep 0 of the RK2 step on d_P, results into scratch):
// ms[0] flux kernels, ms[1] EMF kernel, ms[2] update+inversion kernel, ms[3] one
// bound_prim, ms[4] post_fixup, each averaged over `reps` launches with CUDA events on
// the context stream.  d_P is not modified.
extern "C" int harm_b200_time_stages(harm_ctx* c, int precision, int guess, const double* d_P, double dt, int reps,
                                     double* ms) {
  static const double CUf[4] = {1.0, 0.0, 0.5, 0.0};
  static const double Cun[4] = {0.0, 0.0, 0.0, 0.0};
  Dims d = dims_of(c->g);
  Phys ph = phys_of(c->g);
  if (reps < 1) reps = 1;
  cudaEvent_t ev[6];
  for (int q = 0; q < 6; q++) CK(cudaEventCreate(&ev[q]));
  c->h_scal[0] = dt;
  CK(cudaMemcpyAsync(c->d_dt, c->h_scal, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  for (int q = 0; q < 5; q++) ms[q] = 0.0;
  StepCoef sc;
  sc.CUf0 = CUf[0]; sc.CUf2 = CUf[2]; sc.Cun0 = Cun[0]; sc.Cun1 = Cun[1]; sc.Cun2 = Cun[2];
  sc.finalstep = 0; sc.guess = guess;
  long long ncell = (long long)d.n1 * d.n2 * d.n3;
  FaceBox b1 = face_box(d, 1), b2 = face_box(d, 2), b3 = face_box(d, 3);
  long long nc = (long long)(d.n1 + 1) * (d.n2 + 1) * (d.n3 > 1 ? d.n3 + 1 : 1);
  for (int r = 0; r < reps; r++) {
    CK(cudaEventRecord(ev[0], c->stream));
    if (precision == HARM_PREC_FP64) {
      k_flux<1, double, double><<<nblk(b1.n), 256, 0, c->stream>>>(d, ph, b1, d_P, c->d_geom, c->d_F[0], c->d_dtslots);
      k_flux<2, double, double><<<nblk(b2.n), 256, 0, c->stream>>>(d, ph, b2, d_P, c->d_geom, c->d_F[1], c->d_dtslots + 1);
      if (d.n3 > 1) k_flux<3, double, double><<<nblk(b3.n), 256, 0, c->stream>>>(d, ph, b3, d_P, c->d_geom, c->d_F[2], c->d_dtslots + 2);
      CK(cudaEventRecord(ev[1], c->stream));
      k_emf<double, double><<<nblk(nc), 256, 0, c->stream>>>(d, c->d_F[0], c->d_F[1], c->d_F[2], c->d_geom, c->d_emf);
      CK(cudaEventRecord(ev[2], c->stream));
      k_update<double><<<nblk(ncell), 256, 0, c->stream>>>(d, ph, sc, c->d_dt, d_P, d_P, c->d_pk, c->d_pflag, c->d_F[0],
                                                           c->d_F[1], c->d_F[2], c->d_emf, c->d_geom, c->d_conn,
                                                           c->d_aux, c->d_mlp, nullptr);
    } else {
      k_flux<1, float, float><<<nblk(b1.n), 256, 0, c->stream>>>(d, ph, b1, d_P, c->d_geomf, c->d_Ff[0], c->d_dtslots);
      k_flux<2, float, float><<<nblk(b2.n), 256, 0, c->stream>>>(d, ph, b2, d_P, c->d_geomf, c->d_Ff[1], c->d_dtslots + 1);
      if (d.n3 > 1) k_flux<3, float, float><<<nblk(b3.n), 256, 0, c->stream>>>(d, ph, b3, d_P, c->d_geomf, c->d_Ff[2], c->d_dtslots + 2);
      CK(cudaEventRecord(ev[1], c->stream));
      k_emf<float, float><<<nblk(nc), 256, 0, c->stream>>>(d, c->d_Ff[0], c->d_Ff[1], c->d_Ff[2], c->d_geomf, c->d_emff);
      CK(cudaEventRecord(ev[2], c->stream));
      k_update<float><<<nblk(ncell), 256, 0, c->stream>>>(d, ph, sc, c->d_dt, d_P, d_P, c->d_pk, c->d_pflag, c->d_Ff[0],
                                                          c->d_Ff[1], c->d_Ff[2], c->d_emff, c->d_geom, c->d_conn,
                                                          c->d_aux, c->d_mlp, nullptr);
    }
    c->launches += (d.n3 > 1 ? 5 : 4);
    CK(cudaEventRecord(ev[3], c->stream));
    if (harm_b200_bound(c, c->d_pk)) return 1;
    CK(cudaEventRecord(ev[4], c->stream));
    if (harm_b200_post_fixup(c, c->d_pk, c->d_pflag)) return 1;
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
  for (int q = 0; q < 6; q++) cudaEventDestroy(ev[q]);
  return 0;
}
