// harm_common.cuh -- shared structures, device helpers and kernel templates of the step.
//
// The kernel templates are instantiated per arithmetic path in separate translation units:
//   harm_path_fp64.cu   FP64 path, compiled without FMA contraction (-fmad=false) so that
//                       every FP64 operation is the IEEE operation the C restatement
//                       performs, in the same order;
//   harm_path_mixed.cu  mixed path (FP32 reconstruction/HLL/CT, FP64 update and
//                       inversion), compiled with contraction.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include <stdio.h>
#include <string.h>
#include "harm_b200.h"
#include "harm_device.cuh"
#include "harm_invert.cuh"
#include "harm_mlp.cuh"
#include "harm_weno_f32x2.cuh"
#include "harm_ctx.cuh"

using namespace hb;

// HARM_TU: a tag that keeps the kernel template instantiations of translation units compiled
// with different arithmetic flags apart (the FP64 path is built twice: without and with FMA
// contraction); every kernel template takes it as its last, defaulted, parameter.
#ifndef HARM_TU
#define HARM_TU 0
#endif

int hb_seterr(const char* what, cudaError_t e);
// HARM's [k][j][i][pl] layout -> [pl][k][j][i], planes [k0, k1) (harm_layout.cu)
int hp_harm_to_soa(harm_ctx* c, const double* aos, double* soa, int k0, int k1);
#define CK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return hb_seterr(#call, e_); \
  } while (0)

// Raise kernel `fn`'s dynamic shared-memory limit to `smem` bytes on the current device, once
// per device.  `done` is that kernel's own set of devices already raised (one bit per device
// index, so indices of 64 and above are refused); host threads that drive different devices
// may call this concurrently (the attribute write itself is idempotent).
static inline cudaError_t raise_smem_limit_once(std::atomic<unsigned long long>& done, const void* fn, int smem) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  const unsigned long long bit = 1ull << dev;
  if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

// ------------------------------------------------------------------ indexing helpers

struct Dims {
  int n1, n2, n3, ng, ng3, n1e, n2e, n3e;
  size_t plane, cells;
};

static inline Dims dims_of(const harm_grid& g) {
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
  int laxf;  // fluxmethod LAXF instead of HLL
};

static inline Phys phys_of(const harm_grid& g) {
  Phys p;
  p.gam = g.gam; p.cour = g.cour; p.gammamax = g.gammamax; p.gammafail = g.gammafail;
  p.defcon = g.defcon; p.safe = g.safe;
  p.dx1 = g.dx[1]; p.dx2 = g.dx[2]; p.dx3 = g.dx[3];
  p.laxf = (g.fluxmethod == HARM_FLUX_LAXF);
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

struct FixRec {
  long long id;
  double v[5];
  int flag;  // the cell's flag after the fix
};

// Cell tiles of the per-cell kernels: a block of 256 threads covers TI consecutive i times TK
// consecutive k at one j, so the per-(i,j) metric and connection records a block reads serve
// TK cells each and come from L1 instead of L2, while rows of TI consecutive i keep the state
// loads coalesced.  TI = 256 / TK; lti < 0 selects one thread per cell in i-fastest order.
struct CellTile {
  int lti, ltk;  // log2 TI, log2 TK
};
static inline CellTile cell_tile(int n3, int ltk_max) {
  CellTile ct;
  ct.ltk = 0;
  while (ct.ltk < ltk_max && (2 << ct.ltk) <= n3) ct.ltk++;
  ct.lti = 8 - ct.ltk;
  return ct;
}
static inline CellTile cell_linear() {
  CellTile ct;
  ct.lti = -1;
  ct.ltk = 0;
  return ct;
}
static inline dim3 cell_grid(int n1, int n2, int n3, CellTile ct) {
  if (ct.lti < 0) return dim3((unsigned)(((long long)n1 * n2 * n3 + 255) / 256), 1, 1);
  return dim3((n1 + (1 << ct.lti) - 1) >> ct.lti, n2, (n3 + (1 << ct.ltk) - 1) >> ct.ltk);
}
__device__ __forceinline__ dim3 cell_grid_dev(const Dims& d, CellTile ct) {
  if (ct.lti < 0) return dim3((unsigned)(((long long)d.n1 * d.n2 * d.n3 + 255) / 256), 1, 1);
  return dim3((d.n1 + (1 << ct.lti) - 1) >> ct.lti, d.n2, (d.n3 + (1 << ct.ltk) - 1) >> ct.ltk);
}
// this thread's active cell (i, j, k) in tile (tx, ty, tz); false past the grid's edge
__device__ __forceinline__ bool tile_cell(int n1, int n2, int n3, CellTile ct, int tx, int ty, int tz, int& i, int& j,
                                          int& k) {
  if (ct.lti < 0) {
    const long long t = (long long)tx * 256 + threadIdx.x;
    i = (int)(t % n1);
    const long long r = t / n1;
    j = (int)(r % n2);
    k = (int)(r / n2);
    return t < (long long)n1 * n2 * n3;
  }
  i = (tx << ct.lti) + (int)(threadIdx.x & ((1u << ct.lti) - 1));
  k = (tz << ct.ltk) + (int)(threadIdx.x >> ct.lti);
  j = ty;
  return i < n1 && k < n3;
}

static inline unsigned int nblk(long long n, int bs = 256) { return (unsigned int)((n + bs - 1) / bs); }

// ------------------------------------------------------------------ flux kernel

// Face box of direction DIR (active-relative, inclusive): faces bounding active cells in
// DIR, one transverse ghost layer on each side of every other direction with n>1.
struct FaceBox {
  int lo[3], hi[3], cnt[3];
  long long n;
};

static inline FaceBox face_box(const Dims& d, int dir) {
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

// ------------------------------------------------------------------ tiled flux kernel
//
// One block of 256 threads = a tile of A = 32 faces of direction DIR times NT = 8 transverse
// lines, consecutive threads along i so that every global load is coalesced.  VB primitives
// at a time (all 8 in FP32, 4 in FP64) are staged in shared memory with the stencil halo along
// DIR; the block then computes every cell's reconstruction once (MC slope, para4, the WENO5
// weights and then the edge values, or PARALINE's edges after a pass that computes each
// staged cell's V and total pressure and each edge cell's flattening coefficient), three
// barriers per group instead of three per primitive.
// Each thread keeps the two states of its own face and evaluates states, fluxes, wave speeds
// and the HLL flux of that face.
template <int LIM>
struct ReconGeom;
template <>
struct ReconGeom<HARM_LIM_MC> {
  static constexpr int H = 2, X = 1;  // staged cells below / above the tile's faces
};
template <>
struct ReconGeom<HARM_LIM_PARA> {
  static constexpr int H = 3, X = 2;
};
template <>
struct ReconGeom<HARM_LIM_WENO5> {
  // an edge cell c needs the lower-order fractions of c-1 .. c+1, which need the weights of
  // c-3 .. c+3, which need the cells c-5 .. c+5
  static constexpr int H = 6, X = 5;
};
template <>
struct ReconGeom<HARM_LIM_PARALINE> {
  static constexpr int H = 4, X = 3;  // para edges need cells -2..2, the flattener -3..3
};

template <int LIM, typename T>
struct FluxTile {
  static constexpr int A = 32;                                 // threads (faces) along DIR
  static constexpr int NT = 8;                                 // transverse lines
  static constexpr int H = ReconGeom<LIM>::H;
  static constexpr int VB = (sizeof(T) == 4) ? 8 : 4;          // primitives per stage
  // faces a tile can hold along DIR: one more than its threads, so that the last tile of a
  // sweep of n*A + 1 faces (a grid of n*A cells) takes the last face itself instead of a tile
  // row of one face; the tile's threads tid < NT compute that face, one per line
  static constexpr int AF = A + 1;
  static constexpr int NL = AF + H + ReconGeom<LIM>::X;        // staged cells along DIR
  static constexpr int NW = (LIM == HARM_LIM_WENO5) ? 4 : 0;   // WENO5: 3 weights + SMONO per cell
  static constexpr int PLANE = NL * NT;               // staged values of one primitive
  static constexpr int PE = (AF + 1) * NT;             // edge values: cells H-1 .. H+AF-1
  static constexpr int PW = (NL - 4) * NT;             // WENO5 weights: cells 2 .. NL-3
  static constexpr int NF = (LIM == HARM_LIM_PARALINE) ? 1 : 0;  // PARALINE: V, P, Fi planes
  static constexpr int ND = (LIM == HARM_LIM_WENO5) ? 1 : 0;     // WENO5: dP of the edge cells
  static constexpr size_t smem =
      ((size_t)VB * (PLANE + 2 * PE + NW * PW) + (size_t)NF * (2 * PLANE + PE) + (size_t)ND * PE) * sizeof(T);
  // WENO5's four per-cell line planes of dP (rho, par, veff, upar) live in the edge planes
  // until the edges are written
  static_assert(LIM != HARM_LIM_WENO5 || 2 * VB * PE >= 4 * PLANE, "dP line planes fit the edge planes");
};

// ------------------------------------------------------------------ WENO5BND tile passes
// Shared by k_fluxt and k_fluxt_tma.  Layout helpers: sx(c, t) the staged plane, ex(c, t) the
// edge planes (cells H-1 .. H+A-1), wx(c, t) the weight planes (cells 2 .. NL-3), split(idx,
// c0, nc, v, c, t) the item order.

// dP line quantities of one staged cell into the four line planes tmp[4][PL]
template <int DIR, int PL, typename T>
__device__ __forceinline__ void weno_line_cell(T* tmp, int si, const T* pc, const Geo<T>& g, T gam) {
  T par, veff, upar;
  weno_dp_cell<T>(pc, g, gam, DIR, par, veff, upar);
  tmp[si] = pc[HARM_RHO];
  tmp[PL + si] = par;
  tmp[2 * PL + si] = veff;
  tmp[3 * PL + si] = upar;
}

// dP of the edge cells from the line planes
template <int A, int NT, int H, int PL, typename T, typename SX, typename EX, typename SPLIT>
__device__ __forceinline__ void weno_dp_edges(const T* tmp, T* s_dP, int tid, SX sx, EX ex, SPLIT split) {
  for (int idx = tid; idx < (A + 1) * NT; idx += 256) {
    int v, c, t;
    split(idx, H - 1, A + 1, v, c, t);
    const int i0 = sx(c, t), im = sx(c - 1, t), ip = sx(c + 1, t);
    s_dP[ex(c, t)] = weno_dp<T>(tmp[i0], tmp[PL + i0], tmp[3 * PL + i0], tmp[2 * PL + im], tmp[2 * PL + ip],
                                tmp[3 * PL + im], tmp[3 * PL + ip]);
  }
}

// the lower-order fraction of the cell whose weights are at ws[wx(c, t) * 4]
template <typename T, typename WX>
__device__ __forceinline__ T weno_frac_at(const T* ws, int c, int t, WX wx) {
  const T* w0 = ws + wx(c, t) * 4;
  const T* wm = ws + wx(c - 2, t) * 4;
  const T* wp = ws + wx(c + 2, t) * 4;
  T a[3] = {w0[0], w0[1], w0[2]}, b[3] = {wm[0], wm[1], wm[2]}, e[3] = {wp[0], wp[1], wp[2]};
  return weno_frac<T>(a, b, e);
}

// WENO5BND edges of NV staged primitives: pass 1 the SMONO indicator and the weights of cells
// 2 .. NL-3, barrier, pass 2 the lower-order fraction (raised by dP) and the edges of cells
// H-1 .. H+A-1.  s_dP holds the edge cells' dP and must be ordered before pass 2 by the
// caller's barriers (pass 1 ends with one).
template <int NV, int A, int NT, int H, int NL, int PL, int PE, int PW, typename T, typename SX, typename EX,
          typename WX, typename SPLIT>
__device__ __forceinline__ void weno_tile_edges(const T* s_y, T* s_w, T* s_el, T* s_er, const T* s_dP, int tid,
                                                SX sx, EX ex, WX wx, SPLIT split) {
  if constexpr (sizeof(T) == 4) {
    // FP32: two cells per thread on the packed FP32 pipe (harm_weno_f32x2.cuh)
    constexpr int NU = NV * (NL - 4) * NT, NU2 = (NU + 1) / 2;
    for (int idx = tid; idx < NU2; idx += 256) {
      const int ib = idx + NU2;
      const bool hasb = ib < NU;
      int va, ca, ta, vb, cb, tb;
      split(idx, 2, NL - 4, va, ca, ta);
      split(hasb ? ib : idx, 2, NL - 4, vb, cb, tb);
      const T* ya = s_y + va * PL;
      const T* yb = s_y + vb * PL;
      F2 u5[5];
#pragma unroll
      for (int q = 0; q < 5; q++) u5[q] = f2((float)ya[sx(ca - 2 + q, ta)], (float)yb[sx(cb - 2 + q, tb)]);
      F2 w[3];
      const F2 m = smono_indicator_f2(u5 + 2);
      weno5_cell_weights_f2(u5 + 2, m, w);
      T* wsa = s_w + (va * PW + wx(ca, ta)) * 4;
      T* wsb = s_w + (vb * PW + wx(cb, tb)) * 4;
      float a, b;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        f2split(w[k], a, b);
        wsa[k] = (T)a;
        if (hasb) wsb[k] = (T)b;
      }
      f2split(m, a, b);
      wsa[3] = (T)a;
      if (hasb) wsb[3] = (T)b;
    }
    __syncthreads();
    constexpr int NE = NV * (A + 1) * NT, NE2 = (NE + 1) / 2;
    for (int idx = tid; idx < NE2; idx += 256) {
      const int ib = idx + NE2;
      const bool hasb = ib < NE;
      int va, ca, ta, vb, cb, tb;
      split(idx, H - 1, A + 1, va, ca, ta);
      split(hasb ? ib : idx, H - 1, A + 1, vb, cb, tb);
      const T* ya = s_y + va * PL;
      const T* yb = s_y + vb * PL;
      F2 u5[5];
#pragma unroll
      for (int q = 0; q < 5; q++) u5[q] = f2((float)ya[sx(ca - 2 + q, ta)], (float)yb[sx(cb - 2 + q, tb)]);
      const T* wa = s_w + va * PW * 4;
      const T* wb = s_w + vb * PW * 4;
      F2 w[3], wm[3], wp[3];
#pragma unroll
      for (int k = 0; k < 3; k++) {
        w[k] = f2((float)wa[wx(ca, ta) * 4 + k], (float)wb[wx(cb, tb) * 4 + k]);
        wm[k] = f2((float)wa[wx(ca - 2, ta) * 4 + k], (float)wb[wx(cb - 2, tb) * 4 + k]);
        wp[k] = f2((float)wa[wx(ca + 2, ta) * 4 + k], (float)wb[wx(cb + 2, tb) * 4 + k]);
      }
      const F2 m = f2((float)wa[wx(ca, ta) * 4 + 3], (float)wb[wx(cb, tb) * 4 + 3]);
      F2 f = weno_frac_f2(w, wm, wp);
      const float ssa = weno_dp_strength<float>((float)s_dP[ex(ca, ta)]);
      const float ssb = weno_dp_strength<float>((float)s_dP[ex(cb, tb)]);
      if (ssa > 0.0f || ssb > 0.0f) {  // rare: a momentum-flux jump above 0.25
        float fa, fb;
        f2split(f, fa, fb);
        if (ssa > 0.0f)
          fa = weno_lof<float>(fa, (float)weno_frac_at<T>(wa, ca - 1, ta, wx), (float)weno_frac_at<T>(wa, ca + 1, ta, wx), ssa);
        if (ssb > 0.0f)
          fb = weno_lof<float>(fb, (float)weno_frac_at<T>(wb, cb - 1, tb, wx), (float)weno_frac_at<T>(wb, cb + 1, tb, wx), ssb);
        f = f2(fa, fb);
      }
      F2 yl, yr;
      weno5_edges_f2(u5 + 2, w, f, m, yl, yr);
      float la, lb, ra, rb;
      f2split(yl, la, lb);
      f2split(yr, ra, rb);
      s_el[va * PE + ex(ca, ta)] = (T)la;
      s_er[va * PE + ex(ca, ta)] = (T)ra;
      if (hasb) {
        s_el[vb * PE + ex(cb, tb)] = (T)lb;
        s_er[vb * PE + ex(cb, tb)] = (T)rb;
      }
    }
  } else {
    for (int idx = tid; idx < NV * (NL - 4) * NT; idx += 256) {
      int v, c, t;
      split(idx, 2, NL - 4, v, c, t);
      const T* y = s_y + v * PL;
      T u5[5] = {y[sx(c - 2, t)], y[sx(c - 1, t)], y[sx(c, t)], y[sx(c + 1, t)], y[sx(c + 2, t)]};
      const T m = smono_indicator<T>(u5 + 2);
      T w[3];
      weno5_cell_weights<T>(u5 + 2, m, w);
      T* ws = s_w + (v * PW + wx(c, t)) * 4;
      ws[0] = w[0]; ws[1] = w[1]; ws[2] = w[2]; ws[3] = m;
    }
    __syncthreads();
    for (int idx = tid; idx < NV * (A + 1) * NT; idx += 256) {
      int v, c, t;
      split(idx, H - 1, A + 1, v, c, t);
      const T* y = s_y + v * PL;
      T u5[5] = {y[sx(c - 2, t)], y[sx(c - 1, t)], y[sx(c, t)], y[sx(c + 1, t)], y[sx(c + 2, t)]};
      const T* ws = s_w + v * PW * 4;
      const T* w0 = ws + wx(c, t) * 4;
      T w[3] = {w0[0], w0[1], w0[2]};
      const T m = w0[3];
      T f = weno_frac_at<T>(ws, c, t, wx);
      const T ss = weno_dp_strength<T>(s_dP[ex(c, t)]);
      if (ss > T(0)) f = weno_lof<T>(f, weno_frac_at<T>(ws, c - 1, t, wx), weno_frac_at<T>(ws, c + 1, t, wx), ss);
      T yl, yr;
      weno5_edges<T>(u5 + 2, w, f, m, yl, yr);
      s_el[v * PE + ex(c, t)] = yl;
      s_er[v * PE + ex(c, t)] = yr;
    }
  }
}


// The face physics of k_fluxt: B^DIR continuity, limit_gamma, states, fluxes, wave speeds and
// the HLL flux of one face (flux.c:852, vchar.c:34; LAXF where both speeds vanish or where
// fluxmethod is LAXF, fluxcompute.c:243) into F at `id`; returns cour*dx/ctop.
template <int DIR, typename T, typename GT>
__device__ __forceinline__ double face_hll(const Dims& d, const Phys& ph, const GT* __restrict__ geom,
                                           T* __restrict__ F, size_t id, int ii, int jj, T* pl, T* pr) {
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
  if (!ph.laxf && cmax + cmin != T(0)) {
    const T inv = cmax + cmin;
#pragma unroll
    for (int p = 0; p < NPR; p++) F[(size_t)p * d.cells + id] = ((cmax * Fl[p] + cmin * Fr[p]) - (cmax * cmin) * (Ur[p] - Ul[p])) / inv;
  } else {
#pragma unroll
    for (int p = 0; p < NPR; p++) F[(size_t)p * d.cells + id] = T(0.5) * ((Fl[p] + Fr[p]) - ctop * (Ur[p] - Ul[p]));
  }
  const double dxd = (DIR == 1) ? ph.dx1 : (DIR == 2) ? ph.dx2 : ph.dx3;
  double dtij = ph.cour * dxd / (double)ctop;
  if (!(dtij > 0.0)) dtij = 1.e300;
  return dtij;
}

// HARM_FLUXT_MINB: resident blocks per SM the tiled flux kernel is compiled for (the mixed
// path's FP32 tiles: 3, at most 85 registers with every staging load in flight; the FP64
// tiles: 2, 128 registers with spills, faster than the ~160 registers and 1 block per SM the
// compiler picks on its own); unset, the compiler's choice
#ifdef HARM_FLUXT_MINB
#define HARM_FLUXT_LB __launch_bounds__(256, HARM_FLUXT_MINB)
#else
#define HARM_FLUXT_LB __launch_bounds__(256)
#endif
// DIR 2 and 3 tiles: how far their first line (i) is moved below the face box so that the
// extended index of every tile's first line is a multiple of NT
template <int NT>
__host__ __device__ __forceinline__ int fluxt_tshift(const FaceBox& fb, int ng) {
  static_assert((NT & (NT - 1)) == 0, "NT is a power of two");
  return (fb.lo[0] + ng) & (NT - 1);
}

// L (WENO5, optional): the dP line quantities of every extended cell from k_cellprep,
// [3 (DIR-1) + q][cells] for q = par, veff, upar; where null, the kernel computes them.
template <int DIR, int LIM, typename T, typename GT, int TU = HARM_TU>
__global__ void HARM_FLUXT_LB k_fluxt(Dims d, Phys ph, FaceBox fb, const double* __restrict__ P,
                                               const GT* __restrict__ geom, T* __restrict__ F,
                                               unsigned long long* __restrict__ dtslot,
                                               const T* __restrict__ L = nullptr) {
  using TL = FluxTile<LIM, T>;
  constexpr int A = TL::A, AF = TL::AF, NT = TL::NT, H = TL::H, NL = TL::NL, VB = TL::VB, PL = TL::PLANE, PE = TL::PE, PW = TL::PW;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* s_y = reinterpret_cast<T*>(smem_raw);   // [VB][plane]
  T* s_el = s_y + VB * PL;                    // left edge of each cell, [VB][PE]
  T* s_er = s_el + VB * PE;                   // right edge of each cell, [VB][PE]
  T* s_w = s_er + VB * PE;                    // WENO5 weights and SMONO indicator, [VB][PW][4]
  T* s_V = s_w + VB * PW * TL::NW;            // PARALINE: sqrt(-g) rho u^DIR, [plane]
  T* s_P = s_V + PL;                          // PARALINE: p + b^2/2, [plane]
  T* s_F = s_P + PL;                          // PARALINE: flattening coefficient, [PE]
  T* s_dP = s_w + VB * PW * TL::NW + TL::NF * (2 * PL + PE);  // WENO5: dP of the edge cells, [PE]
  // a plane is [NT][NL] for DIR 1 and [NL][NT] otherwise: the index along i is contiguous
  auto sx = [](int c, int t) -> int { return (DIR == 1) ? t * NL + c : c * NT + t; };
  // edge planes hold cells H-1 .. H+AF-1, weight planes cells 2 .. NL-3, in the same layout
  auto ex = [](int c, int t) -> int { return (DIR == 1) ? t * (AF + 1) + c - (H - 1) : (c - (H - 1)) * NT + t; };
  auto wx = [](int c, int t) -> int { return (DIR == 1) ? t * (NL - 4) + c - 2 : (c - 2) * NT + t; };
  // item idx over VB x nc cells (from c0) x NT lines, fastest along i
  auto split = [](int idx, int c0, int nc, int& v, int& c, int& t) {
    if (DIR == 1) {
      c = c0 + idx % nc;
      int r = idx / nc;
      t = r % NT;
      v = r / NT;
    } else {
      t = idx % NT;
      int r = idx / NT;
      c = c0 + r % nc;
      v = r / nc;
    }
  };
  const int tid = threadIdx.x;
  // tile origin in active-relative face coordinates, and this thread's face.  For DIR 2 and 3
  // the NT lines are consecutive i: their origin is moved down to an extended i that is a
  // multiple of NT (fluxt_tshift), so that each staged row of NT values starts on a 32-byte
  // sector (FP32 rows: one sector, FP64 rows: two); the lanes below the face box do no face.
  int l0, t0, o, lme, tme;
  if (DIR == 1) {
    l0 = blockIdx.x * A + fb.lo[0]; t0 = blockIdx.y * NT + fb.lo[1]; o = blockIdx.z + fb.lo[2];
    lme = tid % A; tme = tid / A;
  } else if (DIR == 2) {
    t0 = blockIdx.x * NT + fb.lo[0] - fluxt_tshift<NT>(fb, d.ng); l0 = blockIdx.y * A + fb.lo[1]; o = blockIdx.z + fb.lo[2];
    lme = tid / NT; tme = tid % NT;
  } else {
    t0 = blockIdx.x * NT + fb.lo[0] - fluxt_tshift<NT>(fb, d.ng); l0 = blockIdx.y * A + fb.lo[2]; o = blockIdx.z + fb.lo[1];
    lme = tid / NT; tme = tid % NT;
  }
  const int lhi = fb.hi[DIR - 1];
  const int thi = (DIR == 1) ? fb.hi[1] : fb.hi[0];
  const int tlo = (DIR == 1) ? fb.lo[1] : fb.lo[0];
  const bool valid = (l0 + lme <= lhi) && (t0 + tme <= thi) && (t0 + tme >= tlo);
  // extended-grid extents along DIR and along the transverse tile axis
  const int ngL = (DIR == 3) ? d.ng3 : d.ng;
  const int nLe = (DIR == 1) ? d.n1e : (DIR == 2) ? d.n2e : d.n3e;
  const int nTe = (DIR == 1) ? d.n2e : d.n1e;
  auto cell_index = [&](int lext, int text) -> size_t {
    if (DIR == 1) return cidx(d, lext, text, o + d.ng3);
    if (DIR == 2) return cidx(d, text, lext, o + d.ng3);
    return cidx(d, text, o + d.ng, lext);
  };
  if constexpr (LIM == HARM_LIM_PARALINE) {
    // get_V_and_P (interpline.c:2964) of every staged cell from all its primitives and the
    // cell-centre metric, then the flattening coefficient of each edge cell; the first
    // staging group's barrier orders the s_F writes before the edge loop reads them
    const T gam = (T)ph.gam;
    for (int idx = tid; idx < PL; idx += 256) {
      int v, cl, ct;
      split(idx, 0, NL, v, cl, ct);
      const int lext = min(max(l0 - H + cl + ngL, 0), nLe - 1);
      const int text = min(max(t0 + ct + d.ng, 0), nTe - 1);
      const size_t cid = cell_index(lext, text);
      T pc[NPR];
#pragma unroll
      for (int p = 0; p < NPR; p++) pc[p] = (T)__ldg(P + (size_t)p * d.cells + cid);
      const int ii = (DIR == 1) ? lext : text, jj = (DIR == 1) ? text : (DIR == 2) ? lext : o + d.ng;
      Geo<T> g;
      load_geo<T, GT>(geom + (size_t)HARM_LOC_CENT * HARM_NGF * d.plane, d.plane, (size_t)jj * d.n1e + ii, g);
      State<T> q;
      get_state<T>(pc, g, gam, q);
      s_V[sx(cl, ct)] = g.gdet * pc[HARM_RHO] * q.ucon[DIR];
      T pt = q.pressure;
      pt += T(0.5) * q.bsq;
      s_P[sx(cl, ct)] = pt;
    }
    __syncthreads();
    for (int idx = tid; idx < (AF + 1) * NT; idx += 256) {
      int v, c, t;
      split(idx, H - 1, AF + 1, v, c, t);
      T vv[7], pp[7];
#pragma unroll
      for (int q = 0; q < 7; q++) {
        vv[q] = s_V[sx(c - 3 + q, t)];
        pp[q] = s_P[sx(c - 3 + q, t)];
      }
      s_F[ex(c, t)] = paraline_fi<T>(vv, pp);
    }
  }
  // WENO5: the line quantities of dP (compute_df_line_new interpline.c:3557) of the staged
  // cells H-2 .. H+A (the edge cells and their neighbours along DIR), from all the cell's
  // primitives and the cell-centre metric, into the edge planes, then dP of each edge cell.
  // From L where the cell pass computed them; otherwise here: with all primitives staged at
  // once (FP32) from the staged tile below, else (FP64, two groups) loaded here.
  constexpr int DPC = AF + 3;  // cells with line quantities per line
  auto weno_line = [&](int cl, int ct, const T* pc) {
    const int lext = min(max(l0 - H + cl + ngL, 0), nLe - 1);
    const int text = min(max(t0 + ct + d.ng, 0), nTe - 1);
    const int ii = (DIR == 1) ? lext : text, jj = (DIR == 1) ? text : (DIR == 2) ? lext : o + d.ng;
    Geo<T> g;
    load_geo<T, GT>(geom + (size_t)HARM_LOC_CENT * HARM_NGF * d.plane, d.plane, (size_t)jj * d.n1e + ii, g);
    weno_line_cell<DIR, PL, T>(s_el, sx(cl, ct), pc, g, (T)ph.gam);
  };
  const bool dp_from_L = (LIM == HARM_LIM_WENO5) && (L != nullptr);
  if constexpr (LIM == HARM_LIM_WENO5) {
    if (dp_from_L) {
      const T* Lq = L + (size_t)3 * (DIR - 1) * d.cells;
      for (int idx = tid; idx < DPC * NT; idx += 256) {
        int v, cl, ct;
        split(idx, H - 2, DPC, v, cl, ct);
        const int lext = min(max(l0 - H + cl + ngL, 0), nLe - 1);
        const int text = min(max(t0 + ct + d.ng, 0), nTe - 1);
        const size_t cid = cell_index(lext, text);
        const int si = sx(cl, ct);
        s_el[si] = (T)__ldg(P + (size_t)HARM_RHO * d.cells + cid);
        s_el[PL + si] = __ldg(Lq + cid);
        s_el[2 * PL + si] = __ldg(Lq + d.cells + cid);
        s_el[3 * PL + si] = __ldg(Lq + 2 * d.cells + cid);
      }
      __syncthreads();
      weno_dp_edges<AF, NT, H, PL, T>(s_el, s_dP, tid, sx, ex, split);
    } else if constexpr (VB < NPR) {
      for (int idx = tid; idx < DPC * NT; idx += 256) {
        int v, cl, ct;
        split(idx, H - 2, DPC, v, cl, ct);
        const int lext = min(max(l0 - H + cl + ngL, 0), nLe - 1);
        const int text = min(max(t0 + ct + d.ng, 0), nTe - 1);
        const size_t cid = cell_index(lext, text);
        T pc[NPR];
#pragma unroll
        for (int p = 0; p < NPR; p++) pc[p] = (T)__ldg(P + (size_t)p * d.cells + cid);
        weno_line(cl, ct, pc);
      }
      __syncthreads();
      weno_dp_edges<AF, NT, H, PL, T>(s_el, s_dP, tid, sx, ex, split);
    }
  }
  T pl[NPR], pr[NPR];
  __shared__ T s_xl[NPR * NT], s_xr[NPR * NT];  // edge values of the tile's face A
#pragma unroll
  for (int p0 = 0; p0 < NPR; p0 += VB) {
    if (p0 > 0) __syncthreads();
    // stage VB primitives (the tile's cells and the halo along DIR; cells past the grid's
    // edge are clamped: they only feed faces outside the face box).  Fully unrolled, so
    // that all of a thread's loads are in flight together.
#pragma unroll
    for (int idx = tid; idx < VB * PL; idx += 256) {
      int v, cl, ct;
      split(idx, 0, NL, v, cl, ct);
      int lext = min(max(l0 - H + cl + ngL, 0), nLe - 1);
      int text = min(max(t0 + ct + d.ng, 0), nTe - 1);
      s_y[v * PL + sx(cl, ct)] = (T)__ldg(P + (size_t)(p0 + v) * d.cells + cell_index(lext, text));
    }
    __syncthreads();
    if constexpr (LIM == HARM_LIM_WENO5) {
      if constexpr (VB == NPR) {
        if (!dp_from_L) {
          for (int idx = tid; idx < DPC * NT; idx += 256) {
            int v, cl, ct;
            split(idx, H - 2, DPC, v, cl, ct);
            T pc[NPR];
#pragma unroll
            for (int p = 0; p < NPR; p++) pc[p] = s_y[p * PL + sx(cl, ct)];
            weno_line(cl, ct, pc);
          }
          __syncthreads();
          weno_dp_edges<AF, NT, H, PL, T>(s_el, s_dP, tid, sx, ex, split);
        }
      }
      weno_tile_edges<VB, AF, NT, H, NL, PL, PE, PW, T>(s_y, s_w, s_el, s_er, s_dP, tid, sx, ex, wx, split);
    } else if (LIM == HARM_LIM_PARA) {
      for (int idx = tid; idx < VB * (AF + 1) * NT; idx += 256) {
        int v, c, t;
        split(idx, H - 1, AF + 1, v, c, t);
        const T* y = s_y + v * PL;
        T u5[5] = {y[sx(c - 2, t)], y[sx(c - 1, t)], y[sx(c, t)], y[sx(c + 1, t)], y[sx(c + 2, t)]};
        T yl, yr;
        para4_cell<T>(u5 + 2, yl, yr);
        s_el[v * PE + ex(c, t)] = yl;
        s_er[v * PE + ex(c, t)] = yr;
      }
    } else if (LIM == HARM_LIM_PARALINE) {
      for (int idx = tid; idx < VB * (AF + 1) * NT; idx += 256) {
        int v, c, t;
        split(idx, H - 1, AF + 1, v, c, t);
        const T* y = s_y + v * PL;
        T u5[5] = {y[sx(c - 2, t)], y[sx(c - 1, t)], y[sx(c, t)], y[sx(c + 1, t)], y[sx(c + 2, t)]};
        T yl, yr;
        paraline_cell<T>(u5 + 2, s_F[ex(c, t)], yl, yr);
        s_el[v * PE + ex(c, t)] = yl;
        s_er[v * PE + ex(c, t)] = yr;
      }
    } else {
      for (int idx = tid; idx < VB * (AF + 1) * NT; idx += 256) {
        int v, c, t;
        split(idx, H - 1, AF + 1, v, c, t);
        const T* y = s_y + v * PL;
        const T y0 = y[sx(c, t)];
        T dq = mc_slope(y[sx(c - 1, t)], y0, y[sx(c + 1, t)]);
        s_el[v * PE + ex(c, t)] = y0 - T(0.5) * dq;
        s_er[v * PE + ex(c, t)] = y0 + T(0.5) * dq;
      }
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < VB; v++) {
      pl[p0 + v] = s_er[v * PE + ex(H + lme - 1, tme)];
      pr[p0 + v] = s_el[v * PE + ex(H + lme, tme)];
    }
    if (tid < NT) {  // the edge values of face A of line tid, read back by the same thread below
#pragma unroll
      for (int v = 0; v < VB; v++) {
        s_xl[(p0 + v) * NT + tid] = s_er[v * PE + ex(H + A - 1, tid)];
        s_xr[(p0 + v) * NT + tid] = s_el[v * PE + ex(H + A, tid)];
      }
    }
  }
  double dtij = 1.e300;
  if (valid) {
    const int lext = l0 + lme + ngL, text = t0 + tme + d.ng;
    const size_t id = cell_index(lext, text);
    int ii, jj;
    if (DIR == 1) { ii = lext; jj = text; }
    else if (DIR == 2) { ii = text; jj = lext; }
    else { ii = text; jj = o + d.ng; }
    dtij = face_hll<DIR, T, GT>(d, ph, geom, F, id, ii, jj, pl, pr);
  }
  {
    // the tile's face A (the sweep's last face), on line tid, by the threads tid < NT, from
    // the edge values each of them kept from every staging group
    if (tid < NT && l0 + A == lhi && t0 + tid <= thi && t0 + tid >= tlo) {
#pragma unroll
      for (int v = 0; v < NPR; v++) {
        pl[v] = s_xl[v * NT + tid];
        pr[v] = s_xr[v * NT + tid];
      }
      const int lext = l0 + A + ngL, text = t0 + tid + d.ng;
      const size_t id = cell_index(lext, text);
      int ii, jj;
      if (DIR == 1) { ii = lext; jj = text; }
      else if (DIR == 2) { ii = text; jj = lext; }
      else { ii = text; jj = o + d.ng; }
      dtij = fmin(dtij, face_hll<DIR, T, GT>(d, ph, geom, F, id, ii, jj, pl, pr));
    }
  }
  // block minimum and one atomic per block
  __shared__ double red[8];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) dtij = fmin(dtij, __shfl_xor_sync(0xffffffffu, dtij, off));
  if ((tid & 31) == 0) red[tid >> 5] = dtij;
  __syncthreads();
  if (tid < 32) {
    double v = (tid < 8) ? red[tid] : 1.e300;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
    if (tid == 0 && v < 1.e300) atomicMin(dtslot, dbl_bits(v));
  }
}

// tiles along a sweep of n faces, with room for one more face in the last tile
// (FluxTile::AF): ceil((n - 1) / A), whose last tile holds 2 .. A+1 faces
template <int LIM, typename T>
static inline int fluxt_tiles(int n) {
  constexpr int A = FluxTile<LIM, T>::A;
  static_assert(FluxTile<LIM, T>::AF == A + 1, "the last tile holds up to A+1 faces");
  return n >= 2 ? (n - 1 + A - 1) / A : 1;
}

template <int DIR, int LIM, typename T>
static inline dim3 fluxt_grid(const FaceBox& fb, int ng) {
  constexpr int NT = FluxTile<LIM, T>::NT;
  if (DIR == 1) return dim3(fluxt_tiles<LIM, T>(fb.cnt[0]), (fb.cnt[1] + NT - 1) / NT, fb.cnt[2]);
  const int nx = (fb.cnt[0] + fluxt_tshift<NT>(fb, ng) + NT - 1) / NT;
  if (DIR == 2) return dim3(nx, fluxt_tiles<LIM, T>(fb.cnt[1]), fb.cnt[2]);
  return dim3(nx, fluxt_tiles<LIM, T>(fb.cnt[2]), fb.cnt[1]);
}

// the face box restricted to active-relative k indices [klo, khi] (index 2: k for every
// direction, the face index along k for DIR 3); false when nothing is left
static inline bool face_box_k(FaceBox b, int klo, int khi, FaceBox* out) {
  klo = (klo > b.lo[2]) ? klo : b.lo[2];
  khi = (khi < b.hi[2]) ? khi : b.hi[2];
  if (klo > khi) return false;
  b.lo[2] = klo;
  b.hi[2] = khi;
  b.cnt[2] = khi - klo + 1;
  b.n = (long long)b.cnt[0] * b.cnt[1] * b.cnt[2];
  *out = b;
  return true;
}

// The cell pass of a WENO5 flux stage: the dP line quantities (par, veff, upar of
// compute_df_line_new interpline.c:3557) of every extended cell of planes [k0, k1), for the
// three directions, from one evaluation of the cell's state (get_state) in the arithmetic
// type T of the flux tiles; L[3 (dir-1) + q][cells].  The tiles of the three directions
// read them instead of evaluating the state of each staged cell once per direction.
template <typename T, typename GT, int TU = HARM_TU>
__global__ void __launch_bounds__(256) k_cellprep(Dims d, Phys ph, const double* __restrict__ P,
                                                  const GT* __restrict__ geom, T* __restrict__ L, int k0, int k1) {
  const long long n = (long long)(k1 - k0) * d.plane;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const size_t id = (size_t)k0 * d.plane + (size_t)t;
  const size_t c2 = (size_t)t % d.plane;
  T pc[NPR];
#pragma unroll
  for (int p = 0; p < NPR; p++) pc[p] = (T)__ldg(P + (size_t)p * d.cells + id);
  Geo<T> g;
  load_geo<T, GT>(geom + (size_t)HARM_LOC_CENT * HARM_NGF * d.plane, d.plane, c2, g);
  State<T> q;
  get_state<T>(pc, g, (T)ph.gam, q);
#pragma unroll
  for (int dir = 1; dir <= 3; dir++) {
    T par, veff, upar;
    weno_dp_of_state<T>(pc, g, q, dir, par, veff, upar);
    L[(size_t)(3 * (dir - 1) + 0) * d.cells + id] = par;
    L[(size_t)(3 * (dir - 1) + 1) * d.cells + id] = veff;
    L[(size_t)(3 * (dir - 1) + 2) * d.cells + id] = upar;
  }
}

template <typename T, typename GT>
static inline cudaError_t launch_cellprep(const Dims& d, const Phys& ph, const double* P, const GT* geom, T* L, int k0,
                                          int k1, cudaStream_t st) {
  const long long n = (long long)(k1 - k0) * d.plane;
  if (n <= 0) return cudaSuccess;
  k_cellprep<T, GT><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d, ph, P, geom, L, k0, k1);
  return cudaGetLastError();
}

// launch k_fluxt<DIR, LIM, T, GT>; the first launch of an instantiation on a device raises
// its dynamic shared-memory limit where the tile needs more than 48 KB (FP32 WENO5: 63 KB)
template <int DIR, int LIM, typename T, typename GT>
static inline cudaError_t launch_fluxt(const Dims& d, const Phys& ph, const FaceBox& fb, const double* P,
                                       const GT* geom, T* F, unsigned long long* dtslot, cudaStream_t st,
                                       const T* L = nullptr) {
  constexpr size_t smem = FluxTile<LIM, T>::smem;
  if (smem > 48 * 1024) {
    static std::atomic<unsigned long long> raised{0};  // per instantiation
    cudaError_t e = raise_smem_limit_once(raised, (const void*)k_fluxt<DIR, LIM, T, GT>, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_fluxt<DIR, LIM, T, GT><<<fluxt_grid<DIR, LIM, T>(fb, d.ng), 256, smem, st>>>(d, ph, fb, P, geom, F, dtslot, L);
  return cudaGetLastError();
}

// The three flux directions of one substep while the state is still arriving in k-slabs
// (SlabWait): after each slab's copy, the x1 and x2 faces of its planes (their stencils stay in
// the plane) and every row of x3 tiles (A faces along k) whose staged planes have all arrived.
// Same kernels and results as the whole-grid launches.
// L (WENO5, optional): the cell pass's output buffer; each slab's cell pass runs once the
// slab has arrived, before the tiles that stage its planes.
template <int LIM, typename T, typename GT>
static inline cudaError_t launch_flux_slabs(const Dims& d, const Phys& ph, const double* pb, const GT* geom, T* F1,
                                            T* F2, T* F3, unsigned long long* slots, cudaStream_t st,
                                            const SlabWait& sw, unsigned long long& launches, T* L = nullptr) {
  constexpr int A = FluxTile<LIM, T>::A, X = ReconGeom<LIM>::X;
  const FaceBox b1 = face_box(d, 1), b2 = face_box(d, 2), b3 = face_box(d, 3);
  int f3 = b3.lo[2];  // first x3 face not launched yet
  cudaError_t e;
  for (int s = 0; s < sw.nslab; s++) {
    if ((e = cudaStreamWaitEvent(st, sw.ev[s], 0)) != cudaSuccess) return e;
    const int resident = (s + 1) * sw.planes;  // planes [0, resident) are on the device
    const int klo = s * sw.planes - d.ng3, khi = resident - 1 - d.ng3;
    if (sw.aos && hp_harm_to_soa(sw.ctx, sw.aos, sw.soa, s * sw.planes, resident < d.n3e ? resident : d.n3e))
      return cudaErrorLaunchFailure;
    if (L) {
      const int k1 = resident < d.n3e ? resident : d.n3e;
      if ((e = launch_cellprep<T, GT>(d, ph, pb, geom, L, s * sw.planes, k1, st)) != cudaSuccess) return e;
      launches++;
    }
    FaceBox sb;
    if (face_box_k(b1, klo, khi, &sb)) {
      if ((e = launch_fluxt<1, LIM, T, GT>(d, ph, sb, pb, geom, F1, slots + 0, st, L)) != cudaSuccess) return e;
      launches++;
    }
    if (face_box_k(b2, klo, khi, &sb)) {
      if ((e = launch_fluxt<2, LIM, T, GT>(d, ph, sb, pb, geom, F2, slots + 1, st, L)) != cudaSuccess) return e;
      launches++;
    }
    // x3 tile rows: a row of faces f0 .. last stages planes up to last + ng3 + X (clamped);
    // a row of tiles with room for one more face takes the sweep's last face when it is the
    // only one left after it
    while (d.n3 > 1 && f3 <= b3.hi[2]) {
      int last = f3 + A - 1;
      if (b3.hi[2] - last == 1) last = b3.hi[2];
      int top = last + d.ng3 + X;
      if (top > d.n3e - 1) top = d.n3e - 1;
      if (top >= resident && s + 1 < sw.nslab) break;
      if (face_box_k(b3, f3, last, &sb)) {
        if ((e = launch_fluxt<3, LIM, T, GT>(d, ph, sb, pb, geom, F3, slots + 2, st, L)) != cudaSuccess) return e;
        launches++;
      }
      f3 = last + 1;
    }
  }
  return cudaSuccess;
}

// ------------------------------------------------------------------ EMF kernel

template <typename T, typename GT, int TU = HARM_TU>
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

// RK coefficients of one substep (setup_rktimestep step_ch.c:1171) and, where the caller keeps
// the step's conserved arrays (harm_b200_advance_u), their device pointers: ui = primtoU(p_i)
// is written, uf and ucum are read (from the second substep on) and written, as
// advance_standard's dUtoU does (advance.c:2046).  Without them the substep's uf and ucum
// start from zero, which is exact for the coefficient sets that never carry them (TIMEORDER 1,
// the RK2 midpoint).
struct StepCoef {
  double CUf0, CUf1, CUf2, Cun0, Cun1, Cun2;
  int finalstep;
  int guess;
  int first;        // the step's first substep (uf and ucum start from zero)
  double* ui;       // NULL: no conserved arrays
  double* uf;
  double* ucum;
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
    // a face's field flux is the average of its two edge EMFs, added in FP64: the sum of two
    // FP32 values is exact there, so the flux-CT telescoping that keeps the corner div B at
    // round-off holds exactly (rounded FP32 sums leave ~1e-7 of |EMF| per step in div B)
    if (p == HARM_B1) {
      f1a = 0.0; f1b = 0.0;
      f2a = -0.5 * ((double)E(e3, ii, jj, kk) + (double)E(e3, ii + 1, jj, kk));
      f2b = -0.5 * ((double)E(e3, ii, jj + 1, kk) + (double)E(e3, ii + 1, jj + 1, kk));
      if (has3) {
        f3a = 0.5 * ((double)E(e2, ii, jj, kk) + (double)E(e2, ii + 1, jj, kk));
        f3b = 0.5 * ((double)E(e2, ii, jj, kk + 1) + (double)E(e2, ii + 1, jj, kk + 1));
      }
    } else if (p == HARM_B2) {
      f1a = 0.5 * ((double)E(e3, ii, jj, kk) + (double)E(e3, ii, jj + 1, kk));
      f1b = 0.5 * ((double)E(e3, ii + 1, jj, kk) + (double)E(e3, ii + 1, jj + 1, kk));
      f2a = 0.0; f2b = 0.0;
      if (has3) {
        f3a = -0.5 * ((double)E(e1, ii, jj, kk) + (double)E(e1, ii, jj + 1, kk));
        f3b = -0.5 * ((double)E(e1, ii, jj, kk + 1) + (double)E(e1, ii, jj + 1, kk + 1));
      }
    } else {
      f1a = -0.5 * ((double)E(e2, ii, jj, kk) + (double)E(e2, ii, jj, kq));
      f1b = -0.5 * ((double)E(e2, ii + 1, jj, kk) + (double)E(e2, ii + 1, jj, kq));
      f2a = 0.5 * ((double)E(e1, ii, jj, kk) + (double)E(e1, ii, jj, kq));
      f2b = 0.5 * ((double)E(e1, ii, jj + 1, kk) + (double)E(e1, ii, jj + 1, kq));
      f3a = 0.0; f3b = 0.0;
    }
  }
  double d1 = -(f1b - f1a) * idx1;
  double d2 = -(f2b - f2a) * idx2;
  double d3 = has3 ? -(f3b - f3a) * idx3 : 0.0;
  return d1 + d2 + d3;
}

// connection source (source_conn): dU^{UU+l} = gdet [ T^j_k Gamma^k_{l j} - rho u^j Gamma^t_{l j} ]
template <bool LDG = true>
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
      for (int k = 0; k < 4; k++) s += mhd[j][k] * tab_ld<LDG>(conn + (size_t)((k * 4 + l) * 4 + j) * plane + c2);
#pragma unroll
    for (int j = 0; j < 4; j++) s += -pr[HARM_RHO] * q.ucon[j] * tab_ld<LDG>(conn + (size_t)((0 * 4 + l) * 4 + j) * plane + c2);
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

// Conserved update of one substep: U_i = primtoU(p_i), flux divergence (field fluxes from
// the EMFs), connection source of p_b, RK combination; U (UEVOLVE) to global memory.
// (One pass, in the reference's order of operations: the FP64 path.)
// minimum resident blocks per SM the FP64 kernels are compiled for (register budget)
#ifndef HARM_CONSERVED_BLOCKS
#define HARM_CONSERVED_BLOCKS 2
#endif
// log2 of the k extent of the cell tiles (0: whole i rows, one thread per cell in order)
#ifndef HARM_CONSERVED_LTK
#define HARM_CONSERVED_LTK 0
#endif
#ifndef HARM_INVERT_LTK
#define HARM_INVERT_LTK 4
#endif
#ifndef HARM_INVERT_BLOCKS
#define HARM_INVERT_BLOCKS 3
#endif

// STAGE (the conserved-update kernels): cell tiles of 16 i x 16 k at one j (CellTile lti = 4);
// the connection and CENT metric records of the tile's 16 (i,j) columns are staged in shared
// memory once per block (each serves 16 cells) instead of being loaded by every cell, which
// also frees the registers the per-cell loads held in flight.
constexpr int kStageTI = 16;
constexpr int kStageF = 64 + HARM_NGF;  // connection entries, then the metric record
template <bool STAGE>
__device__ __forceinline__ void stage_conn_geom(const Dims& d, const double* __restrict__ geom,
                                                const double* __restrict__ conn, double* s_tab) {
  if constexpr (STAGE) {
    const int i0 = blockIdx.x * kStageTI, jj0 = blockIdx.y + d.ng;
    for (int e = threadIdx.x; e < kStageF * kStageTI; e += blockDim.x) {
      const int f = e / kStageTI, il = e % kStageTI;
      const int ii0 = min(i0 + il, d.n1 - 1) + d.ng;
      const size_t c = (size_t)jj0 * d.n1e + ii0;
      s_tab[e] = (f < 64) ? __ldg(conn + (size_t)f * d.plane + c) : __ldg(geom + (size_t)(f - 64) * d.plane + c);
    }
    __syncthreads();
  }
}

template <typename T, bool STAGE = false, int TU = HARM_TU>
__global__ void __launch_bounds__(256, HARM_CONSERVED_BLOCKS) k_conserved(Dims d, Phys ph, StepCoef sc, const double* __restrict__ dtp,
                                                      const double* __restrict__ pi, const double* __restrict__ pb,
                                                      const T* __restrict__ F1, const T* __restrict__ F2,
                                                      const T* __restrict__ F3, const T* __restrict__ emf,
                                                      const double* __restrict__ geom, const double* __restrict__ conn,
                                                      double* __restrict__ Uout, CellTile ct) {
  __shared__ double s_tab[STAGE ? kStageF * kStageTI : 1];
  int i, j, k;
  const bool ok = tile_cell(d.n1, d.n2, d.n3, ct, blockIdx.x, blockIdx.y, blockIdx.z, i, j, k);
  stage_conn_geom<STAGE>(d, geom, conn, s_tab);
  if (!ok) return;
  int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
  const size_t id = cidx(d, ii, jj, kk), c2 = (size_t)jj * d.n1e + ii;
  const int il = i & (kStageTI - 1);
  Geo<double> g;
  if constexpr (STAGE) load_geo<double, double, false>(s_tab + 64 * kStageTI, kStageTI, il, g);
  else load_geo<double, double>(geom, d.plane, c2, g);
  double pr[NPR];
#pragma unroll
  for (int p = 0; p < NPR; p++) pr[p] = pi[(size_t)p * d.cells + id];
  State<double> q;
  get_state<double>(pr, g, ph.gam, q);
  double Ui[NPR];
  primtoflux<double>(pr, q, 0, g, g.gdet, Ui);
#pragma unroll
  for (int p = 0; p < NPR; p++) pr[p] = pb[(size_t)p * d.cells + id];
  get_state<double>(pr, g, ph.gam, q);
  double dUg[NPR];
  if constexpr (STAGE) source_conn<false>(pr, q, g, s_tab, kStageTI, il, dUg);
  else source_conn(pr, q, g, conn, d.plane, c2, dUg);
  const double idx1 = 1.0 / ph.dx1, idx2 = 1.0 / ph.dx2, idx3 = 1.0 / ph.dx3;
  const double dt = *dtp;
#pragma unroll
  for (int p = 0; p < NPR; p++) {
    const size_t q = (size_t)p * d.cells + id;
    double dU = dU_cell<T>(d, ii, jj, kk, p, F1, F2, F3, emf, idx1, idx2, idx3);
    if (sc.uf) {  // UFSET, ucum += UCUMUPDATE (global.stepch.h:1, :10) with the caller's arrays
      const double ufo = sc.first ? 0.0 : sc.uf[q], uco = sc.first ? 0.0 : sc.ucum[q];
      const double Uf = sc.CUf0 * Ui[p] + sc.CUf1 * ufo + sc.CUf2 * dt * (dU + dUg[p]);
      const double uc = uco + (sc.Cun0 * Ui[p] + sc.Cun1 * dt * (dU + dUg[p]) + sc.Cun2 * Uf);
      sc.ui[q] = Ui[p];
      sc.uf[q] = Uf;
      sc.ucum[q] = uc;
      Uout[q] = sc.finalstep ? uc : Uf;
    } else {
      double Uf = sc.CUf0 * Ui[p] + sc.CUf2 * dt * (dU + dUg[p]);
      double ucum = sc.Cun0 * Ui[p] + sc.Cun1 * dt * (dU + dUg[p]) + sc.Cun2 * Uf;
      Uout[q] = sc.finalstep ? ucum : Uf;
    }
  }
}

// The conserved update in two passes (the mixed path): k_conserved_src writes
// U = a Ui + b dt dUg (U_i = primtoU(p_i), dUg the connection source of p_b) and
// k_conserved_div adds b dt dU (the flux divergence), with a = CUf0, b = CUf2 for an
// intermediate substep and a = Cun0 + Cun2 CUf0, b = Cun1 + Cun2 CUf2 for the final one
// (Uf and ucum of k_conserved expanded: both are linear in U_i and dU + dUg).  Each pass needs
// fewer registers than the single kernel, so both run at a higher occupancy.
#ifndef HARM_CONSERVED_SRC_BLOCKS
#define HARM_CONSERVED_SRC_BLOCKS 3
#endif
__device__ __forceinline__ void conserved_ab(const StepCoef& sc, double& a, double& b) {
  a = sc.finalstep ? sc.Cun0 + sc.Cun2 * sc.CUf0 : sc.CUf0;
  b = sc.finalstep ? sc.Cun1 + sc.Cun2 * sc.CUf2 : sc.CUf2;
}

template <typename T, bool STAGE, int TU = HARM_TU>
__global__ void __launch_bounds__(256, HARM_CONSERVED_SRC_BLOCKS) k_conserved_src(Dims d, Phys ph, StepCoef sc, const double* __restrict__ dtp,
                                                      const double* __restrict__ pi, const double* __restrict__ pb,
                                                      const double* __restrict__ geom, const double* __restrict__ conn,
                                                      double* __restrict__ Uout, CellTile ct) {
  __shared__ double s_tab[STAGE ? kStageF * kStageTI : 1];
  int i, j, k;
  const bool ok = tile_cell(d.n1, d.n2, d.n3, ct, blockIdx.x, blockIdx.y, blockIdx.z, i, j, k);
  stage_conn_geom<STAGE>(d, geom, conn, s_tab);
  if (!ok) return;
  int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
  const size_t id = cidx(d, ii, jj, kk), c2 = (size_t)jj * d.n1e + ii;
  const int il = i & (kStageTI - 1);
  Geo<double> g;
  if constexpr (STAGE) load_geo<double, double, false>(s_tab + 64 * kStageTI, kStageTI, il, g);
  else load_geo<double, double>(geom, d.plane, c2, g);
  double pr[NPR];
#pragma unroll
  for (int p = 0; p < NPR; p++) pr[p] = pi[(size_t)p * d.cells + id];
  State<double> q;
  get_state<double>(pr, g, ph.gam, q);
  double Ui[NPR];
  primtoflux<double>(pr, q, 0, g, g.gdet, Ui);
#pragma unroll
  for (int p = 0; p < NPR; p++) pr[p] = pb[(size_t)p * d.cells + id];
  get_state<double>(pr, g, ph.gam, q);
  double dUg[NPR];
  if constexpr (STAGE) source_conn<false>(pr, q, g, s_tab, kStageTI, il, dUg);
  else source_conn(pr, q, g, conn, d.plane, c2, dUg);
  if (sc.uf) {
    // the caller's conserved arrays: uf and ucum without the flux divergence, which
    // k_conserved_div adds (both are linear in it)
    const double dt = *dtp;
#pragma unroll
    for (int p = 0; p < NPR; p++) {
      const size_t q = (size_t)p * d.cells + id;
      const double ufo = sc.first ? 0.0 : sc.uf[q], uco = sc.first ? 0.0 : sc.ucum[q];
      const double Uf = sc.CUf0 * Ui[p] + sc.CUf1 * ufo + sc.CUf2 * dt * dUg[p];
      sc.ui[q] = Ui[p];
      sc.uf[q] = Uf;
      sc.ucum[q] = uco + (sc.Cun0 * Ui[p] + sc.Cun1 * dt * dUg[p] + sc.Cun2 * Uf);
    }
    return;
  }
  double a, b;
  conserved_ab(sc, a, b);
  const double bdt = b * *dtp;
#pragma unroll
  for (int p = 0; p < NPR; p++) Uout[(size_t)p * d.cells + id] = a * Ui[p] + bdt * dUg[p];
}

template <typename T, int TU = HARM_TU>
__global__ void __launch_bounds__(256) k_conserved_div(Dims d, Phys ph, StepCoef sc, const double* __restrict__ dtp,
                                                      const T* __restrict__ F1, const T* __restrict__ F2,
                                                      const T* __restrict__ F3, const T* __restrict__ emf,
                                                      double* __restrict__ U, CellTile ct) {
  int i, j, k;
  if (!tile_cell(d.n1, d.n2, d.n3, ct, blockIdx.x, blockIdx.y, blockIdx.z, i, j, k)) return;
  int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
  const size_t id = cidx(d, ii, jj, kk);
  const double idx1 = 1.0 / ph.dx1, idx2 = 1.0 / ph.dx2, idx3 = 1.0 / ph.dx3;
  if (sc.uf) {
    const double dt = *dtp, bf = sc.CUf2 * dt, bc = (sc.Cun1 + sc.Cun2 * sc.CUf2) * dt;
#pragma unroll
    for (int p = 0; p < NPR; p++) {
      const size_t q = (size_t)p * d.cells + id;
      const double dU = dU_cell<T>(d, ii, jj, kk, p, F1, F2, F3, emf, idx1, idx2, idx3);
      const double uf = sc.uf[q] + bf * dU, uc = sc.ucum[q] + bc * dU;
      sc.uf[q] = uf;
      sc.ucum[q] = uc;
      U[q] = sc.finalstep ? uc : uf;
    }
    return;
  }
  double a, b;
  conserved_ab(sc, a, b);
  const double bdt = b * *dtp;
#pragma unroll
  for (int p = 0; p < NPR; p++) {
    const double dU = dU_cell<T>(d, ii, jj, kk, p, F1, F2, F3, emf, idx1, idx2, idx3);
    U[(size_t)p * d.cells + id] += bdt * dU;
  }
}

// Inversion of one substep, common path: the hot Newton inversion of U with p_b as guess,
// then, when no floor acts, limit_gamma (the end of fixup1zone).  Cells whose hot inversion
// failed, or whose density or internal energy falls below a floor, are appended to a list
// and finished by k_invert_rare, so that the rarely taken branches (cold inversion, the
// floor re-inversion) neither diverge warps nor enlarge the register footprint here.
// PATH distinguishes the instantiation of each arithmetic path's translation unit.
// GUESS: the Newton iteration starts from wpg[t] (the learned start, k_mlp_guess) where it is
// positive; a cell whose learned start does not converge starts again from the
// previous-state W', exactly as without GUESS (counted in stats[2]).
// The common-path inversion of active cell (i, j, k), as described above; w is the learned
// start (GUESS), iters_d and fb_d receive the Newton iterations and the fallback count.
template <bool GUESS>
__device__ __forceinline__ void invert_cell(const Dims& d, const Phys& ph, const double* __restrict__ U,
                                            const double* __restrict__ pb, double* __restrict__ pf,
                                            int8_t* __restrict__ pflag, const double* __restrict__ geom,
                                            const double* __restrict__ aux, unsigned int* __restrict__ rare,
                                            unsigned int* __restrict__ nrare, int i, int j, int k, double w,
                                            double& iters_d, double& fb_d) {
  const long long t = i + (long long)d.n1 * (j + (long long)d.n2 * k);  // active-cell index
  int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
  const size_t id = cidx(d, ii, jj, kk), c2 = (size_t)jj * d.n1e + ii;
  Geo<double> g;
  load_geo<double, double>(geom, d.plane, c2, g);
  double Ugf[NPR], pr[NPR];
#pragma unroll
  for (int p = 0; p < NPR; p++) { Ugf[p] = U[(size_t)p * d.cells + id] * g.igdet; pr[p] = pb[(size_t)p * d.cells + id]; }
  int8_t flag = 0;
  int it = 0;
  if (GUESS) {
    JonSetup s;
    jon_prepare(false, Ugf, g, pr, ph.gam, ph.gammafail, s);
    jon_solve(s, (w > 0.0) ? w : s.Wp_prev, pr, flag, it);
    if (flag != 0 && w > 0.0) {  // the learned start did not converge: the plain start
      fb_d += 1.0;
      jon_solve(s, s.Wp_prev, pr, flag, it);
    }
  } else {
    utoprim_jon(false, Ugf, g, flag, pr, ph.gam, ph.gammafail, it, false, 0.0);
  }
  iters_d += (double)it;
  bool defer = (flag != 0);
  if (!defer) {
    double rhofl = __ldg(aux + (size_t)HARM_AUX_RHOFLOOR * d.plane + c2);
    double ufl = __ldg(aux + (size_t)HARM_AUX_UFLOOR * d.plane + c2);
    rhofl = (rhofl < kSMALL) ? kSMALL : rhofl;
    ufl = (ufl < kSMALL) ? kSMALL : ufl;
    defer = (rhofl > pr[HARM_RHO]) || (ufl > pr[HARM_UU]);
    if (!defer) limit_gamma<double>(ph.gammamax, pr, g);
  }
  if (defer) {
    unsigned int slot = atomicAdd(nrare, 1u);
    rare[slot] = (unsigned int)t;
  }
  pflag[id] = flag;
#pragma unroll
  for (int p = 0; p < NPR; p++) pf[(size_t)p * d.cells + id] = pr[p];
}

template <int PATH, bool GUESS = false>
__global__ void __launch_bounds__(256, HARM_INVERT_BLOCKS) k_invert(Dims d, Phys ph, const double* __restrict__ U,
                                                   const double* __restrict__ pb, double* __restrict__ pf,
                                                   int8_t* __restrict__ pflag, const double* __restrict__ geom,
                                                   const double* __restrict__ aux, unsigned int* __restrict__ rare,
                                                   unsigned int* __restrict__ nrare, double* __restrict__ stats,
                                                   CellTile ct, const double* __restrict__ wpg = nullptr) {
  double iters_d = 0.0, fb_d = 0.0;
  int i, j, k;
  if (tile_cell(d.n1, d.n2, d.n3, ct, blockIdx.x, blockIdx.y, blockIdx.z, i, j, k)) {
    const double w = GUESS ? wpg[i + (long long)d.n1 * (j + (long long)d.n2 * k)] : 0.0;
    invert_cell<GUESS>(d, ph, U, pb, pf, pflag, geom, aux, rare, nrare, i, j, k, w, iters_d, fb_d);
  }
  if (stats) {
    warp_add_atomic(iters_d, stats + 0);
    if (GUESS) warp_add_atomic(fb_d, stats + 2);
  }
}

// The gated learned start, first kernel: the plain inversion of k_invert (the same operations
// from the previous-state W'), except that a cell whose first Newton step exceeds `gate` of
// the convergence scale (its previous state is a poor start: a floored cell, a shock, a cold
// start) stops after that step and is appended to the list `hard`; k_invert_hard then solves
// it from the learned start.  Every other cell's result is the plain path's, bit for bit.
template <int PATH>
__global__ void __launch_bounds__(256, HARM_INVERT_BLOCKS) k_invert_gated(Dims d, Phys ph, const double* __restrict__ U,
                                                   const double* __restrict__ pb, double* __restrict__ pf,
                                                   int8_t* __restrict__ pflag, const double* __restrict__ geom,
                                                   const double* __restrict__ aux, unsigned int* __restrict__ rare,
                                                   unsigned int* __restrict__ nrare, double* __restrict__ stats,
                                                   CellTile ct, double gate, unsigned int* __restrict__ hard,
                                                   unsigned int* __restrict__ nhard) {
  double iters_d = 0.0;
  int i, j, k;
  if (tile_cell(d.n1, d.n2, d.n3, ct, blockIdx.x, blockIdx.y, blockIdx.z, i, j, k)) {
    const long long t = i + (long long)d.n1 * (j + (long long)d.n2 * k);
    const int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
    const size_t id = cidx(d, ii, jj, kk), c2 = (size_t)jj * d.n1e + ii;
    Geo<double> g;
    load_geo<double, double>(geom, d.plane, c2, g);
    double Ugf[NPR], pr[NPR];
#pragma unroll
    for (int p = 0; p < NPR; p++) { Ugf[p] = U[(size_t)p * d.cells + id] * g.igdet; pr[p] = pb[(size_t)p * d.cells + id]; }
    int8_t flag = 0;
    int it = 0;
    JonSetup s;
    jon_prepare(false, Ugf, g, pr, ph.gam, ph.gammafail, s);
    const bool poor = jon_solve<true>(s, s.Wp_prev, pr, flag, it, nullptr, gate);
    iters_d = (double)it;
    if (poor) {
      hard[atomicAdd(nhard, 1u)] = (unsigned int)t;
    } else {
      bool defer = (flag != 0);
      if (!defer) {
        double rhofl = __ldg(aux + (size_t)HARM_AUX_RHOFLOOR * d.plane + c2);
        double ufl = __ldg(aux + (size_t)HARM_AUX_UFLOOR * d.plane + c2);
        rhofl = (rhofl < kSMALL) ? kSMALL : rhofl;
        ufl = (ufl < kSMALL) ? kSMALL : ufl;
        defer = (rhofl > pr[HARM_RHO]) || (ufl > pr[HARM_UU]);
        if (!defer) limit_gamma<double>(ph.gammamax, pr, g);
      }
      if (defer) rare[atomicAdd(nrare, 1u)] = (unsigned int)t;
      pflag[id] = flag;
#pragma unroll
      for (int p = 0; p < NPR; p++) pf[(size_t)p * d.cells + id] = pr[p];
    }
  }
  if (stats) warp_add_atomic(iters_d, stats + 0);
}

// The learned start of the inversion, one kernel before k_invert: per cell the
// alpha-scaled invariants of U (compute_setup_quantities), the features, the network on the
// tensor cores (per warp, mma.sync BF16 with FP32 accumulation) and W' = D exp(log(W'/D) +
// start_bias) into wpg (-1 where the prediction is not a positive finite number).  A
// persistent grid walks the cells in tiles of 256, so the packed network is copied to shared
// memory once per block.  Kept apart from the Newton iteration so that each kernel runs at
// its own occupancy (this one needs few registers, the FP64 iteration many).
template <int PATH>
#ifndef HARM_MLP_GUESS_BLOCKS
#define HARM_MLP_GUESS_BLOCKS 3
#endif
__global__ void __launch_bounds__(256, HARM_MLP_GUESS_BLOCKS) k_mlp_guess(Dims d, const double* __restrict__ U,
                                                      const double* __restrict__ geom, double* __restrict__ wpg,
                                                      const MlpPacked* __restrict__ mlp, CellTile ct) {
  __shared__ MlpPacked sm;
  __shared__ MlpWarpScratch wsc[8];
  mlp_load_packed(sm, mlp);
  __syncthreads();
  const dim3 gg = cell_grid_dev(d, ct);
  const int gx = (int)gg.x;
  const long long ntiles = (long long)gg.x * gg.y * gg.z;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int i, j, k;
    const long long rest = tile / gx;
    const bool valid = tile_cell(d.n1, d.n2, d.n3, ct, (int)(tile % gx), (int)(rest % gg.y), (int)(rest / gg.y), i, j, k);
    const long long t = i + (long long)d.n1 * (j + (long long)d.n2 * k);
    float f[MLP_IN];
    double D = 0.0;
    if (valid) {
      int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
      const size_t id = cidx(d, ii, jj, kk), c2 = (size_t)jj * d.n1e + ii;
      Geo<double> g;
      load_geo<double, double>(geom, d.plane, c2, g);
      double Ua[NPR];
#pragma unroll
      for (int p = 0; p < NPR; p++) Ua[p] = g.alpha * (U[(size_t)p * d.cells + id] * g.igdet);
      InvC c;
      double Qtcon[4], Bcon[4];
      inv_invariants(Ua, g, c, Qtcon, Bcon);
      mlp_features(c, g, f);
      D = c.D;
    }
    float y[MLP_OUT];
    mlp_warp_eval(sm, wsc[threadIdx.x >> 5], f, valid, y);
    if (valid) {
      const double wp = D * exp((double)y[0] + (double)sm.start_bias);
      wpg[t] = (wp > 0.0 && isfinite(wp)) ? wp : -1.0;
    }
  }
}

// Inversion, rare path over the listed cells: the cold fallback of a failed hot inversion
// (trycoldinversion utoprimgen.c:594), then fixup1zone (fixup.c:561) with its floor
// re-inversion.  p_f holds the hot result, p_b the guess the hot inversion started from.
template <int PATH>
__global__ void __launch_bounds__(128) k_invert_rare(Dims d, Phys ph, const double* __restrict__ U,
                                                     const double* __restrict__ pb, double* __restrict__ pf,
                                                     int8_t* __restrict__ pflag, const double* __restrict__ geom,
                                                     const double* __restrict__ aux, const unsigned int* __restrict__ rare,
                                                     const unsigned int* __restrict__ nrare, double* __restrict__ stats) {
  const unsigned int n = *nrare;
  for (unsigned int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    long long t = rare[s];
    int i = (int)(t % d.n1);
    long long r = t / d.n1;
    int j = (int)(r % d.n2), k = (int)(r / d.n2);
    int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
    const size_t id = cidx(d, ii, jj, kk), c2 = (size_t)jj * d.n1e + ii;
    Geo<double> g;
    load_geo<double, double>(geom, d.plane, c2, g);
    double pr[NPR];
#pragma unroll
    for (int p = 0; p < NPR; p++) pr[p] = pf[(size_t)p * d.cells + id];
    int8_t flag = pflag[id];
    int it = 0;
    double fails = 0.0;
    if (flag) {
      fails = 1.0;
      double Ugf[NPR], prcold[NPR];
#pragma unroll
      for (int p = 0; p < NPR; p++) { Ugf[p] = U[(size_t)p * d.cells + id] * g.igdet; prcold[p] = pb[(size_t)p * d.cells + id]; }
      double pr0uu = prcold[HARM_UU];
      int8_t cflag = 0;
      utoprim_jon(true, Ugf, g, cflag, prcold, ph.gam, ph.gammafail, it, false, 0.0);
      if (cflag <= 0) {
#pragma unroll
        for (int p = 0; p < NPR; p++) pr[p] = prcold[p];
        pr[HARM_UU] = pr0uu;
        flag = HARM_UTOPRIMFAILU2AVG1;
      }
    }
    double floors = (double)fixup1zone(pr, g, __ldg(aux + (size_t)HARM_AUX_RHOFLOOR * d.plane + c2),
                                       __ldg(aux + (size_t)HARM_AUX_UFLOOR * d.plane + c2), ph.gam, ph.gammamax,
                                       ph.gammafail, flag, it);
    pflag[id] = flag;
#pragma unroll
    for (int p = 0; p < NPR; p++) pf[(size_t)p * d.cells + id] = pr[p];
    if (stats) {
      atomicAdd(stats + 0, (double)it);
      if (fails != 0.0) atomicAdd(stats + 3, fails);
      if (floors != 0.0) atomicAdd(stats + 4, floors);
    }
  }
}

// field fluxes of the faces of active cells from the EMFs (for the standalone fluxcalc)
template <typename T, int TU = HARM_TU>
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

