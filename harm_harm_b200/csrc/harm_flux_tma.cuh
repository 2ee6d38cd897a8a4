// harm_flux_tma.cuh -- the FP32 flux kernel with its stencil tiles staged by TMA.
//
// Same tiles and arithmetic as k_fluxt<DIR, LIM, float> (harm_common.cuh), organised as a
// persistent kernel: each block walks the tiles of a direction; one thread loads a tile's
// 8 primitives with a single 4-D cp.async.bulk.tensor (x = i, y = j, z = k, w = primitive,
// zero fill outside the extended grid) completing on an mbarrier, and the load of the next
// tile is in flight while the block converts, reconstructs and evaluates the current one.
// The TMA x coordinate (i) must start on a 16-byte boundary, so the box starts at the even
// i at or below the first staged cell and is one or two doubles wider; the conversion pass
// reads it from that offset.  Requires 16-byte aligned P and an even n1e (the row pitch is a
// multiple of 16 bytes); other layouts use k_fluxt.  Opt-in (HARM_B200_FLUX_STAGING=tma): on
// B200 the staging is not what bounds the flux stage (the WENO5 arithmetic and the face
// physics are), and the tile loop's registers cost occupancy, so k_fluxt is the default.
#pragma once
#include <cuda.h>
#include "harm_async.cuh"
#include "harm_common.cuh"

namespace hbtma {

using hbasync::fence_mbar_init;
using hbasync::fence_proxy_async;
using hbasync::mbar_init;
using hbasync::mbar_wait;
using hbasync::smem_u32;

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// 4-D tiled load into this CTA's own shared memory
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z,
                                            int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}

}  // namespace hbtma

// the TMA box of a tile (doubles): DIR 1: x = NL cells (+1 for the even start, rounded up to
// an even count), y = 8 lines; DIR 2: x = 8 lines + 2, y = NL; DIR 3: x = 8 + 2, z = NL
template <int DIR, int LIM>
struct TmaBox {
  static constexpr int NL = FluxTile<LIM, float>::NL;
  static constexpr int BX = (DIR == 1) ? ((NL + 2) & ~1) : FluxTile<LIM, float>::NT + 2;
  static constexpr int BY = (DIR == 1) ? FluxTile<LIM, float>::NT : (DIR == 2 ? NL : 1);
  static constexpr int BZ = (DIR == 3) ? NL : 1;
  static constexpr int PER_VAR = BX * BY * BZ;
  static constexpr unsigned BYTES = (unsigned)PER_VAR * NPR * 8u;
  static constexpr size_t RAW_BYTES = ((size_t)BYTES + 127) / 128 * 128;
  static constexpr size_t smem = RAW_BYTES + FluxTile<LIM, float>::smem;  // + the float tile buffers
  static_assert((BX * 8) % 16 == 0, "TMA box rows are whole 16-byte units");
};

constexpr unsigned kTmaWaitLimit = 1u << 22;  // polls of the tile's mbarrier before giving up

// blocks per SM the tile's shared memory allows (WENO5: 89 KB -> 2; MC, PPM: <= 48 KB -> 4)
template <int LIM>
struct TmaOcc {
  static constexpr int blocks = (LIM == HARM_LIM_WENO5) ? 2 : 4;
};

template <int DIR, int LIM, typename GT>
__global__ void __launch_bounds__(256, TmaOcc<LIM>::blocks) k_fluxt_tma(Dims d, Phys ph, FaceBox fb, const __grid_constant__ CUtensorMap tmap,
                                                      const GT* __restrict__ geom, float* __restrict__ F,
                                                      unsigned long long* __restrict__ dtslot,
                                                      unsigned int* __restrict__ status) {
  using T = float;
  using TL = FluxTile<LIM, T>;
  using TB = TmaBox<DIR, LIM>;
  constexpr int A = TL::A, AF = TL::AF, NT = TL::NT, H = TL::H, NL = TL::NL, PL = TL::PLANE, PE = TL::PE, PW = TL::PW;
  static_assert(TL::VB == NPR, "the FP32 tile holds all primitives at once");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* raw = reinterpret_cast<double*>(smem_raw);
  T* s_y = reinterpret_cast<T*>(smem_raw + TB::RAW_BYTES);
  T* s_el = s_y + NPR * PL;   // [NPR][PE]
  T* s_er = s_el + NPR * PE;  // [NPR][PE]
  T* s_w = s_er + NPR * PE;   // [NPR][PW][4]
  T* s_dP = s_w + NPR * PW * TL::NW;  // WENO5: dP of the edge cells, [PE]
  __shared__ uint64_t bar;
  __shared__ int s_ok;
  __shared__ double red[8];
  auto sx = [](int c, int t) -> int { return (DIR == 1) ? t * NL + c : c * NT + t; };
  // edge planes hold cells H-1 .. H+AF-1, weight planes cells 2 .. NL-3, in the same layout
  // (this kernel's tiles hold A faces; the edge planes have room for the AF of k_fluxt's)
  auto ex = [](int c, int t) -> int { return (DIR == 1) ? t * (AF + 1) + c - (H - 1) : (c - (H - 1)) * NT + t; };
  auto wx = [](int c, int t) -> int { return (DIR == 1) ? t * (NL - 4) + c - 2 : (c - 2) * NT + t; };
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
  // tiles of this direction: (along i or the transverse i, along j or DIR, along k or j)
  const int gx = (DIR == 1) ? (fb.cnt[0] + A - 1) / A : (fb.cnt[0] + NT - 1) / NT;
  const int gy = (DIR == 1) ? (fb.cnt[1] + NT - 1) / NT : (DIR == 2) ? (fb.cnt[1] + A - 1) / A : (fb.cnt[2] + A - 1) / A;
  const int gz = (DIR == 3) ? fb.cnt[1] : fb.cnt[2];
  const long long ntiles = (long long)gx * gy * gz;
  const int ngL = (DIR == 3) ? d.ng3 : d.ng;
  int lme, tme;
  if (DIR == 1) { lme = tid % A; tme = tid / A; }
  else { lme = tid / NT; tme = tid % NT; }
  // tile origin (active-relative face coordinates) and the TMA box start of tile `tile`
  auto origin = [&](long long tile, int& l0, int& t0, int& o) {
    const int bx = (int)(tile % gx);
    const long long r = tile / gx;
    const int by = (int)(r % gy), bz = (int)(r / gy);
    if (DIR == 1) { l0 = bx * A + fb.lo[0]; t0 = by * NT + fb.lo[1]; o = bz + fb.lo[2]; }
    else if (DIR == 2) { t0 = bx * NT + fb.lo[0]; l0 = by * A + fb.lo[1]; o = bz + fb.lo[2]; }
    else { t0 = bx * NT + fb.lo[0]; l0 = by * A + fb.lo[2]; o = bz + fb.lo[1]; }
  };
  auto box_x = [&](int l0, int t0) -> int {  // first staged i (extended index)
    return (DIR == 1) ? l0 - H + ngL : t0 + d.ng;
  };
  auto issue = [&](long long tile) {
    int l0, t0, o;
    origin(tile, l0, t0, o);
    const int xs = box_x(l0, t0), x0 = xs - (xs & 1);
    int y, z;
    if (DIR == 1) { y = t0 + d.ng; z = o + d.ng3; }
    else if (DIR == 2) { y = l0 - H + ngL; z = o + d.ng3; }
    else { y = o + d.ng; z = l0 - H + ngL; }
    hbtma::fence_proxy_async();
    hbtma::mbar_expect_tx(&bar, TB::BYTES);
    hbtma::tma_load_4d(raw, &tmap, &bar, x0, y, z, 0);
  };
  if (tid == 0) {
    hbtma::mbar_init(&bar, 1);
    hbtma::fence_mbar_init();
  }
  __syncthreads();
  long long tile = blockIdx.x;
  if (tid == 0 && tile < ntiles) issue(tile);
  double dtmin = 1.e300;
  unsigned parity = 0;
  for (; tile < ntiles; tile += gridDim.x) {
    int l0, t0, o;
    origin(tile, l0, t0, o);
    const int xs = box_x(l0, t0), ox = xs & 1;
    if (tid == 0) s_ok = hbtma::mbar_wait(&bar, parity, kTmaWaitLimit) ? 1 : 0;
    __syncthreads();
    if (!s_ok) {  // the tile never arrived: record it and leave (all threads together)
      if (tid == 0) atomicOr(status, 1u);
      return;
    }
    parity ^= 1u;
    // raw doubles -> FP32 tile (cells outside the extended grid arrived as zeros; they only
    // feed faces outside the face box)
    for (int idx = tid; idx < NPR * PL; idx += 256) {
      int v, c, t;
      split(idx, 0, NL, v, c, t);
      const int ri = (DIR == 1) ? t * TB::BX + c + ox : c * TB::BX + t + ox;
      s_y[v * PL + sx(c, t)] = (T)raw[v * TB::PER_VAR + ri];
    }
    __syncthreads();
    if (tid == 0 && tile + gridDim.x < ntiles) issue(tile + gridDim.x);  // the next tile flies now
    if constexpr (LIM == HARM_LIM_WENO5) {
      // dP line quantities of every staged cell from the staged primitives and the
      // cell-centre metric (staged cells outside the extended grid arrived as zeros; their
      // metric is the nearest cell's, and they only feed faces outside the face box)
      const int nLe = (DIR == 1) ? d.n1e : (DIR == 2) ? d.n2e : d.n3e;
      const int nTe = (DIR == 1) ? d.n2e : d.n1e;
      for (int idx = tid; idx < PL; idx += 256) {
        int v, cl, ct;
        split(idx, 0, NL, v, cl, ct);
        T pc[NPR];
#pragma unroll
        for (int p = 0; p < NPR; p++) pc[p] = s_y[p * PL + sx(cl, ct)];
        const int lext = min(max(l0 - H + cl + ngL, 0), nLe - 1);
        const int text = min(max(t0 + ct + d.ng, 0), nTe - 1);
        const int ii = (DIR == 1) ? lext : text, jj = (DIR == 1) ? text : (DIR == 2) ? lext : o + d.ng;
        Geo<T> g;
        load_geo<T, GT>(geom + (size_t)HARM_LOC_CENT * HARM_NGF * d.plane, d.plane, (size_t)jj * d.n1e + ii, g);
        weno_line_cell<DIR, PL, T>(s_el, sx(cl, ct), pc, g, (T)ph.gam);
      }
      __syncthreads();
      weno_dp_edges<AF, NT, H, PL, T>(s_el, s_dP, tid, sx, ex, split);
      weno_tile_edges<NPR, AF, NT, H, NL, PL, PE, PW, T>(s_y, s_w, s_el, s_er, s_dP, tid, sx, ex, wx, split);
    } else if (LIM == HARM_LIM_PARA) {
      for (int idx = tid; idx < NPR * (AF + 1) * NT; idx += 256) {
        int v, c, t;
        split(idx, H - 1, AF + 1, v, c, t);
        const T* y = s_y + v * PL;
        T u5[5] = {y[sx(c - 2, t)], y[sx(c - 1, t)], y[sx(c, t)], y[sx(c + 1, t)], y[sx(c + 2, t)]};
        T yl, yr;
        para4_cell<T>(u5 + 2, yl, yr);
        s_el[v * PE + ex(c, t)] = yl;
        s_er[v * PE + ex(c, t)] = yr;
      }
    } else {
      for (int idx = tid; idx < NPR * (AF + 1) * NT; idx += 256) {
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
    T pl[NPR], pr[NPR];
#pragma unroll
    for (int v = 0; v < NPR; v++) {
      pl[v] = s_er[v * PE + ex(H + lme - 1, tme)];
      pr[v] = s_el[v * PE + ex(H + lme, tme)];
    }
    const int lhi = fb.hi[DIR - 1];
    const int thi = (DIR == 1) ? fb.hi[1] : fb.hi[0];
    if ((l0 + lme <= lhi) && (t0 + tme <= thi)) {
      const int lext = l0 + lme + ngL, text = t0 + tme + d.ng;
      int ii, jj, kk;
      if (DIR == 1) { ii = lext; jj = text; kk = o + d.ng3; }
      else if (DIR == 2) { ii = text; jj = lext; kk = o + d.ng3; }
      else { ii = text; jj = o + d.ng; kk = lext; }
      const double dt = face_hll<DIR, T, GT>(d, ph, geom, F, cidx(d, ii, jj, kk), ii, jj, pl, pr);
      dtmin = fmin(dtmin, dt);
    }
    __syncthreads();  // the tile buffers are rewritten by the next iteration
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) dtmin = fmin(dtmin, __shfl_xor_sync(0xffffffffu, dtmin, off));
  if ((tid & 31) == 0) red[tid >> 5] = dtmin;
  __syncthreads();
  if (tid < 32) {
    double v = (tid < 8) ? red[tid] : 1.e300;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
    if (tid == 0 && v < 1.e300) atomicMin(dtslot, dbl_bits(v));
  }
}
