// harm_mlp_tc.cuh -- the learned start of the inversion on the 5th-generation tensor cores
// (tcgen05), fused with the Newton inversion.
//
// The network is that of harm_mlp.cuh (10 -> 64 -> 64 -> 64 -> 2, SiLU, BF16 weights, FP32
// accumulation).  A warpgroup (128 threads, one cell per thread) evaluates it for a tile of
// 128 cells as four M = 128 MMAs chained through shared memory:
//   - each thread writes its cell's standardised features as one BF16 row of the A operand;
//   - one thread issues tcgen05.mma kind::f16 (A and B from shared memory, D in tensor memory)
//     and tcgen05.commit to the warpgroup's mbarrier;
//   - every thread reads its row of D back with tcgen05.ld (warp q of the warpgroup owns TMEM
//     lanes 32q..32q+31), adds the bias, applies SiLU (layers 1-3 packed with halved weights
//     and biases, as for mma.sync) and writes the BF16 row of the next layer's A operand.
// Operands use the no-swizzle K-major canonical layout: 8-row x 16-byte core matrices of 128
// contiguous bytes; element (r, k) of an operand with KC = K/8 chunks of K lies at byte
// ((r/8)*KC + k/8)*128 + (r%8)*16 + (k%8)*2, so the descriptor's leading-dimension offset
// (between the two 8-element K halves of one MMA) is 128 bytes and its stride-dimension
// offset (between 8-row groups) KC*128 bytes.  The weights are the B operands, W[in][out]
// stored as rows n = out of K = in elements (layer 1: K padded 10 -> 16; layer 4: N padded
// 2 -> 16).  Each warpgroup owns 64 TMEM columns (one 128 x 64 FP32 accumulator, reused by
// every layer).
//
// Waits on the mbarrier are bounded: a thread that gives up sets bit 1 of the device status
// word; the warpgroup's next barrier ORs the threads' give-up flags (bar.red.or), so all 128
// threads stop together; then the warpgroup waits once more, with a bound, for the MMA in
// flight and frees its TMEM.
#pragma once
#include "harm_async.cuh"
#include "harm_common.cuh"

namespace hb {

// byte offsets of the B operands in the packed record
constexpr int TC_W1 = 0;                        // 64 x 16
constexpr int TC_W2 = TC_W1 + 64 * 16 * 2;      // 64 x 64
constexpr int TC_W3 = TC_W2 + 64 * 64 * 2;      // 64 x 64
constexpr int TC_W4 = TC_W3 + 64 * 64 * 2;      // 16 x 64
constexpr int TC_WBYTES = TC_W4 + 16 * 64 * 2;  // 20480

struct MlpTc {
  uint4 w[TC_WBYTES / 16];  // BF16 B operands in the canonical layout
  float bias[MLP_NBIAS];    // b1 b2 b3 b4 (+2 pad)
  float norm[MLP_NNORM];
  float start_bias;
  float pad[3];
};
static_assert(sizeof(MlpTc) % 16 == 0, "packed record is copied as 16-byte words");

// byte offset of element (r, k) in an operand of kc 8-element K chunks
__host__ __device__ __forceinline__ int tc_off(int r, int k, int kc) {
  return ((r >> 3) * kc + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// shared memory of a block of two warpgroups
struct MlpTcBlock {
  MlpTc net;
  uint4 act[2][128 * 64 * 2 / 16];  // per warpgroup: the A operand (128 rows x up to 64 BF16)
  uint64_t mbar[2];
  uint32_t tmem;  // TMEM base address from tcgen05.alloc
};
// a thread's progress through its warpgroup's MMAs
struct TcState {
  unsigned phase;  // parity of the mbarrier phase to wait for next (flipped per layer)
  bool gave_up;    // a wait of this thread ran out
};
constexpr unsigned kTcWaitLimit = 1u << 22;  // polls of an MMA's mbarrier before giving up
constexpr uint32_t kTcCols = 128;            // TMEM columns of a block (64 per warpgroup)

namespace tc {

using hbasync::smem_u32;

// shared-memory matrix descriptor: no swizzle, K-major, the given leading and stride byte
// offsets, descriptor version 1 (bits 46-47)
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor of kind::f16: FP32 D (bits 4-5), BF16 A (7-9) and B (10-12), both
// K-major, N/8 at bits 17-22, M/16 = 8 at bits 24-28
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
// the mbarrier completes one arrival when this thread's MMAs issued so far have completed
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void ld2(uint32_t taddr, uint32_t* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(v[0]), "=r"(v[1]) : "r"(taddr) : "memory");
}
// collective over warp 0
__device__ __forceinline__ void alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// barrier of the 128 threads of warpgroup wg (ids 1 and 2; 0 is __syncthreads) returning the
// OR of their predicates
template <int ID>
__device__ __forceinline__ unsigned bar_red_or(unsigned pred) {
  unsigned v;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, 128, p;\n selp.u32 %0, 1, 0, q;\n}"
      : "=r"(v)
      : "r"(pred), "n"(ID)
      : "memory");
  return v;
}
__device__ __forceinline__ bool wg_sync_any(int wg, bool pred) {
  return (wg == 0 ? bar_red_or<1>((unsigned)pred) : bar_red_or<2>((unsigned)pred)) != 0u;
}

}  // namespace tc

// Block prologue: the packed network into shared memory, the two mbarriers, the TMEM
// columns (warp 0).  Every thread of the block calls it.
__device__ __forceinline__ void mlp_tc_begin(MlpTcBlock& B, const MlpTc* __restrict__ src) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* dst = reinterpret_cast<uint4*>(&B.net);
  for (int i = threadIdx.x; i < (int)(sizeof(MlpTc) / 16); i += blockDim.x) dst[i] = __ldg(s + i);
  if (threadIdx.x == 0) {
    hbasync::mbar_init(&B.mbar[0], 1);
    hbasync::mbar_init(&B.mbar[1], 1);
    hbasync::fence_mbar_init();
  }
  if (threadIdx.x < 32) tc::alloc(&B.tmem, kTcCols);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
}

// Block epilogue: a warpgroup that gave up waits once more (bounded) for its MMA in flight;
// then warp 0 frees the TMEM columns.  Every thread of the block calls it.
__device__ __forceinline__ void mlp_tc_end(MlpTcBlock& B, const TcState& st) {
  const int wg = threadIdx.x >> 7;
  if (tc::wg_sync_any(wg, st.gave_up) && (threadIdx.x & 127) == 0)
    hbasync::mbar_wait(&B.mbar[wg], st.phase ^ 1u, kTcWaitLimit);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (threadIdx.x < 32) tc::dealloc(B.tmem, kTcCols);
}

// standardised features of one cell (zeros for a thread without a cell)
__device__ __forceinline__ void mlp_tc_standardise(const MlpTc& m, const float* f, bool valid, float* x) {
#pragma unroll
  for (int i = 0; i < MLP_IN; i++) x[i] = valid ? (f[i] - m.norm[i]) / m.norm[MLP_IN + i] : 0.0f;
}

// The network for the 128 rows of this thread's warpgroup: x = this row's standardised
// features; y = its de-standardised outputs.  All 128 threads of the warpgroup call it; it
// returns false (for all of them) once a thread of the warpgroup has given up waiting for an
// MMA.
__device__ __forceinline__ bool mlp_tc_eval(MlpTcBlock& B, const float* x, TcState& st,
                                            unsigned int* __restrict__ status, float* y) {
  const int wg = threadIdx.x >> 7, r = threadIdx.x & 127, q = r >> 5;
  unsigned char* act = reinterpret_cast<unsigned char*>(B.act[wg]);
  const uint32_t act_s = tc::smem_u32(act), w_s = tc::smem_u32(B.net.w);
  const uint32_t tcol = B.tmem + 64u * (uint32_t)wg;          // this warpgroup's accumulator
  const uint32_t trow = tcol + ((uint32_t)(q * 32) << 16);     // this warp's TMEM lanes
  {
    uint4 c0, c1;
    c0.x = pack_bf16x2(x[0], x[1]);
    c0.y = pack_bf16x2(x[2], x[3]);
    c0.z = pack_bf16x2(x[4], x[5]);
    c0.w = pack_bf16x2(x[6], x[7]);
    c1.x = pack_bf16x2(x[8], x[9]);
    c1.y = 0u;
    c1.z = 0u;
    c1.w = 0u;
    *reinterpret_cast<uint4*>(act + tc_off(r, 0, 2)) = c0;
    *reinterpret_cast<uint4*>(act + tc_off(r, 8, 2)) = c1;
  }
#pragma unroll 1
  for (int layer = 0; layer < 4; layer++) {
    hbasync::fence_proxy_async();
    tc::fence_before();
    if (tc::wg_sync_any(wg, st.gave_up)) return false;
    if (r == 0) {
      tc::fence_after();
      if (layer == 0) {
        tc::mma_bf16(tcol, tc::sdesc(act_s, 128, 256), tc::sdesc(w_s + TC_W1, 128, 256), tc::idesc_bf16(64), 0u);
      } else {
        const uint32_t wb = w_s + (layer == 1 ? TC_W2 : layer == 2 ? TC_W3 : TC_W4);
        const uint32_t id = tc::idesc_bf16(layer == 3 ? 16 : 64);
#pragma unroll
        for (int ks = 0; ks < 4; ks++)
          tc::mma_bf16(tcol, tc::sdesc(act_s + 256u * ks, 128, 1024), tc::sdesc(wb + 256u * ks, 128, 1024), id,
                       ks > 0 ? 1u : 0u);
      }
      tc::commit(&B.mbar[wg]);
    }
    if (!hbasync::mbar_wait(&B.mbar[wg], st.phase, kTcWaitLimit)) {
      st.gave_up = true;
      atomicOr(status, 2u);
    }
    st.phase ^= 1u;
    tc::fence_after();
    if (layer < 3) {
      const float* b = B.net.bias + layer * MLP_H;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        uint32_t v[32];
        tc::ld16(trow + 32u * h, v);
        tc::ld16(trow + 32u * h + 16u, v + 16);
        tc::wait_ld();
#pragma unroll
        for (int c = 0; c < 4; c++) {
          const int col = 32 * h + 8 * c;
          auto act2 = [&](int e) -> uint32_t {
            return mlp_silu2_bf16(f2(__uint_as_float(v[8 * c + e]), __uint_as_float(v[8 * c + e + 1])) +
                                  f2(b[col + e], b[col + e + 1]));
          };
          uint4 o;
          o.x = act2(0);
          o.y = act2(2);
          o.z = act2(4);
          o.w = act2(6);
          *reinterpret_cast<uint4*>(act + tc_off(r, col, 8)) = o;
        }
      }
    } else {
      uint32_t v[2];
      tc::ld2(trow, v);
      tc::wait_ld();
      const float* nrm = B.net.norm + 2 * MLP_IN;
      const float* b4 = B.net.bias + 3 * MLP_H;
      y[0] = (__uint_as_float(v[0]) + b4[0]) * nrm[MLP_OUT + 0] + nrm[0];
      y[1] = (__uint_as_float(v[1]) + b4[1]) * nrm[MLP_OUT + 1] + nrm[1];
    }
  }
  return true;
}

// Tiles of 128 cells (one per thread of a warpgroup): TI consecutive i times TK consecutive k
// at one j, TI * TK = 128, TK up to 8 (the per-(i,j) metric records serve TK cells each).
struct Tile128 {
  int lti, ltk, gx, gy, gz;
};
static inline Tile128 tile128_of(const Dims& d) {
  Tile128 t;
  t.ltk = 0;
  while (t.ltk < 3 && (2 << t.ltk) <= d.n3) t.ltk++;
  t.lti = 7 - t.ltk;
  t.gx = (d.n1 + (1 << t.lti) - 1) >> t.lti;
  t.gy = d.n2;
  t.gz = (d.n3 + (1 << t.ltk) - 1) >> t.ltk;
  return t;
}
__device__ __forceinline__ bool tile128_cell(const Dims& d, const Tile128& tt, long long tile, int r, int& i, int& j,
                                             int& k) {
  const int tx = (int)(tile % tt.gx);
  const long long rest = tile / tt.gx;
  j = (int)(rest % tt.gy);
  const int tz = (int)(rest / tt.gy);
  i = (tx << tt.lti) + (r & ((1 << tt.lti) - 1));
  k = (tz << tt.ltk) + (r >> tt.lti);
  return i < d.n1 && k < d.n3;
}

// features of active cell (i, j, k) from U (UEVOLVE) and the CENT metric; D: the alpha-scaled
// rest-mass density of the invariants
__device__ __forceinline__ void mlp_cell_features(const Dims& d, const double* __restrict__ U,
                                                  const double* __restrict__ geom, int i, int j, int k, float* f,
                                                  double& D) {
  const int ii = i + d.ng, jj = j + d.ng, kk = k + d.ng3;
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

// Inversion of one substep, common path, with the learned start evaluated in the same kernel:
// per tile of 128 cells, the features of each cell (the alpha-scaled invariants of U, as in
// k_mlp_guess), the network on the tensor cores, then the Newton inversion of invert_cell from
// W' = D exp(log(W'/D) + start_bias).  Persistent: the two warpgroups of a block walk
// alternate tiles, the network is copied to shared memory once per block.
#ifndef HARM_INVERT_TC_BLOCKS
#define HARM_INVERT_TC_BLOCKS HARM_INVERT_BLOCKS
#endif
template <int PATH>
__global__ void __launch_bounds__(256, HARM_INVERT_TC_BLOCKS) k_invert_tc(Dims d, Phys ph, const double* __restrict__ U,
                                                      const double* __restrict__ pb, double* __restrict__ pf,
                                                      int8_t* __restrict__ pflag, const double* __restrict__ geom,
                                                      const double* __restrict__ aux, unsigned int* __restrict__ rare,
                                                      unsigned int* __restrict__ nrare, double* __restrict__ stats,
                                                      Tile128 tt, const MlpTc* __restrict__ mlp,
                                                      unsigned int* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char tc_smem[];
  MlpTcBlock& B = *reinterpret_cast<MlpTcBlock*>(tc_smem);
  mlp_tc_begin(B, mlp);
  const int wg = threadIdx.x >> 7, r = threadIdx.x & 127;
  const long long ntiles = (long long)tt.gx * tt.gy * tt.gz;
  TcState st = {0u, false};
  double iters_d = 0.0, fb_d = 0.0;
  for (long long tile = 2ll * blockIdx.x + wg; tile < ntiles; tile += 2ll * gridDim.x) {
    int i, j, k;
    const bool valid = tile128_cell(d, tt, tile, r, i, j, k);
    float x[MLP_IN];
    double D = 0.0;
    {
      float f[MLP_IN];
      if (valid) mlp_cell_features(d, U, geom, i, j, k, f, D);
      mlp_tc_standardise(B.net, f, valid, x);
    }
    float y[MLP_OUT];
    if (!mlp_tc_eval(B, x, st, status, y)) break;
    if (valid) {
      double w = D * exp((double)y[0] + (double)B.net.start_bias);
      w = (w > 0.0 && isfinite(w)) ? w : -1.0;
      invert_cell<true>(d, ph, U, pb, pf, pflag, geom, aux, rare, nrare, i, j, k, w, iters_d, fb_d);
    }
  }
  mlp_tc_end(B, st);
  if (stats) {
    warp_add_atomic(iters_d, stats + 0);
    warp_add_atomic(fb_d, stats + 2);
  }
}

// The learned start as a kernel of its own (the tensor-core counterpart of k_mlp_guess): per
// tile of 128 cells the features, the network, and W' = D exp(log(W'/D) + start_bias) into
// wpg[t] (-1 where that is not a positive finite number), for k_invert<PATH, true>.
// Persistent, the two warpgroups of a block on alternate tiles.
#ifndef HARM_MLP_TC_BLOCKS
#define HARM_MLP_TC_BLOCKS 4
#endif
template <int PATH>
__global__ void __launch_bounds__(256, HARM_MLP_TC_BLOCKS) k_mlp_guess_tc(Dims d, const double* __restrict__ U,
                                                         const double* __restrict__ geom, double* __restrict__ wpg,
                                                         Tile128 tt, const MlpTc* __restrict__ mlp,
                                                         unsigned int* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char tc_smem[];
  MlpTcBlock& B = *reinterpret_cast<MlpTcBlock*>(tc_smem);
  mlp_tc_begin(B, mlp);
  const int wg = threadIdx.x >> 7, r = threadIdx.x & 127;
  const long long ntiles = (long long)tt.gx * tt.gy * tt.gz;
  TcState st = {0u, false};
  for (long long tile = 2ll * blockIdx.x + wg; tile < ntiles; tile += 2ll * gridDim.x) {
    int i, j, k;
    const bool valid = tile128_cell(d, tt, tile, r, i, j, k);
    float x[MLP_IN];
    double D = 0.0;
    {
      float f[MLP_IN];
      if (valid) mlp_cell_features(d, U, geom, i, j, k, f, D);
      mlp_tc_standardise(B.net, f, valid, x);
    }
    float y[MLP_OUT];
    if (!mlp_tc_eval(B, x, st, status, y)) break;
    if (valid) {
      const double w = D * exp((double)y[0] + (double)B.net.start_bias);
      wpg[i + (long long)d.n1 * (j + (long long)d.n2 * k)] = (w > 0.0 && isfinite(w)) ? w : -1.0;
    }
  }
  mlp_tc_end(B, st);
}

// The learned start inside the inversion kernel with the warp-level mma.sync network: a
// persistent grid walks the cell tiles (k_invert's CellTile order); for each tile every warp
// evaluates the network for its 32 cells (BF16 tensor cores, FP32 accumulation, no block
// barrier), then each thread runs the Newton inversion of its cell from that start.  The
// warps of an SM interleave network phases (tensor and special-function pipes) with Newton
// phases (FP64 pipe), and neither U nor the start makes an extra trip through HBM.
#ifndef HARM_INVERT_MMA_BLOCKS
#define HARM_INVERT_MMA_BLOCKS HARM_INVERT_BLOCKS
#endif
template <int PATH>
__global__ void __launch_bounds__(256, HARM_INVERT_MMA_BLOCKS) k_invert_mma(Dims d, Phys ph, const double* __restrict__ U,
                                                        const double* __restrict__ pb, double* __restrict__ pf,
                                                        int8_t* __restrict__ pflag, const double* __restrict__ geom,
                                                        const double* __restrict__ aux, unsigned int* __restrict__ rare,
                                                        unsigned int* __restrict__ nrare, double* __restrict__ stats,
                                                        CellTile ct, const MlpPacked* __restrict__ mlp) {
  __shared__ MlpPacked sm;
  __shared__ MlpWarpScratch wsc[8];
  mlp_load_packed(sm, mlp);
  __syncthreads();
  const dim3 gg = cell_grid_dev(d, ct);
  const int gx = (int)gg.x;
  const long long ntiles = (long long)gg.x * gg.y * gg.z;
  double iters_d = 0.0, fb_d = 0.0;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    int i, j, k;
    const long long rest = tile / gx;
    const bool valid = tile_cell(d.n1, d.n2, d.n3, ct, (int)(tile % gx), (int)(rest % gg.y), (int)(rest / gg.y), i, j, k);
    float f[MLP_IN];
    double D = 0.0;
    if (valid) mlp_cell_features(d, U, geom, i, j, k, f, D);
    float y[MLP_OUT];
    mlp_warp_eval(sm, wsc[threadIdx.x >> 5], f, valid, y);
    if (valid) {
      double w = D * exp((double)y[0] + (double)sm.start_bias);
      w = (w > 0.0 && isfinite(w)) ? w : -1.0;
      invert_cell<true>(d, ph, U, pb, pf, pflag, geom, aux, rare, nrare, i, j, k, w, iters_d, fb_d);
    }
  }
  if (stats) {
    warp_add_atomic(iters_d, stats + 0);
    warp_add_atomic(fb_d, stats + 2);
  }
}

// k_invert_mma over every active cell: one persistent grid of HARM_INVERT_MMA_BLOCKS blocks
// per SM (fewer when there are fewer tiles)
template <int PATH>
static int launch_invert_mma(harm_ctx* c, const Dims& d, const Phys& ph, const CellTile& ct, const double* pb,
                             double* pf, int8_t* pflag, double* stats) {
  const dim3 g = cell_grid(d.n1, d.n2, d.n3, ct);
  const long long ntiles = (long long)g.x * g.y * g.z;
  const long long cap = (long long)HARM_INVERT_MMA_BLOCKS * c->num_sms;
  const unsigned grid = (unsigned)(ntiles < cap ? ntiles : cap);
  k_invert_mma<PATH><<<grid, 256, 0, c->stream>>>(d, ph, c->d_U, pb, pf, pflag, c->d_geom, c->d_aux, c->d_rare,
                                                   c->d_nrare, stats, ct, reinterpret_cast<const MlpPacked*>(c->d_mlp));
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

// The gated learned start, second kernel: the cells k_invert_gated listed in `hard` (those
// whose previous state is a poor start), with the network inside the inversion kernel as in
// k_invert_mma: per round each warp evaluates the network for 32 listed cells (mma.sync BF16,
// FP32 accumulation), then each thread runs the Newton inversion of its cell from that start;
// a start that does not converge is replaced by the previous-state W' (invert_cell<true>), so
// the result is the plain path's within the Newton tolerance.  The list's length is read on
// the device, so the launch needs no host synchronisation; an empty list returns at once.
// stats[1] receives the number of listed cells.
template <int PATH>
__global__ void __launch_bounds__(256) k_invert_hard(Dims d, Phys ph, const double* __restrict__ U,
                                                     const double* __restrict__ pb, double* __restrict__ pf,
                                                     int8_t* __restrict__ pflag, const double* __restrict__ geom,
                                                     const double* __restrict__ aux, unsigned int* __restrict__ rare,
                                                     unsigned int* __restrict__ nrare, double* __restrict__ stats,
                                                     const unsigned int* __restrict__ hard,
                                                     const unsigned int* __restrict__ nhard,
                                                     const MlpPacked* __restrict__ mlp) {
  __shared__ MlpPacked sm;
  __shared__ MlpWarpScratch wsc[8];
  const unsigned int n = *nhard;
  if (blockIdx.x * 256u >= n) return;  // the same for every thread of the block
  mlp_load_packed(sm, mlp);
  __syncthreads();
  double iters_d = 0.0, fb_d = 0.0, listed = 0.0;
  for (unsigned int base = blockIdx.x * 256u; base < n; base += gridDim.x * 256u) {
    const unsigned int slot = base + threadIdx.x;
    const bool valid = slot < n;
    int i = 0, j = 0, k = 0;
    float f[MLP_IN];
    double D = 0.0;
    if (valid) {
      const long long t = hard[slot];
      i = (int)(t % d.n1);
      const long long r = t / d.n1;
      j = (int)(r % d.n2);
      k = (int)(r / d.n2);
      mlp_cell_features(d, U, geom, i, j, k, f, D);
    }
    float y[MLP_OUT];
    mlp_warp_eval(sm, wsc[threadIdx.x >> 5], f, valid, y);
    if (valid) {
      double w = D * exp((double)y[0] + (double)sm.start_bias);
      w = (w > 0.0 && isfinite(w)) ? w : -1.0;
      invert_cell<true>(d, ph, U, pb, pf, pflag, geom, aux, rare, nrare, i, j, k, w, iters_d, fb_d);
      listed += 1.0;
    }
  }
  if (stats) {
    warp_add_atomic(iters_d, stats + 0);
    warp_add_atomic(listed, stats + 1);
    warp_add_atomic(fb_d, stats + 2);
  }
}

// The gated learned start: k_invert_gated over every active cell, then k_invert_hard over
// the cells it listed (at most one block per 256 cells of the grid, at most two per SM).
template <int PATH>
static int launch_invert_gated(harm_ctx* c, const Dims& d, const Phys& ph, const CellTile& ct, const double* pb,
                               double* pf, int8_t* pflag, double* stats) {
  unsigned int* hard = reinterpret_cast<unsigned int*>(c->d_wpg);  // n1*n2*n3 doubles: room for the list
  CK(cudaMemsetAsync(c->d_nhard, 0, sizeof(unsigned int), c->stream));
  k_invert_gated<PATH><<<cell_grid(d.n1, d.n2, d.n3, ct), 256, 0, c->stream>>>(
      d, ph, c->d_U, pb, pf, pflag, c->d_geom, c->d_aux, c->d_rare, c->d_nrare, stats, ct, c->mlp_gate, hard, c->d_nhard);
  const long long ncell = (long long)d.n1 * d.n2 * d.n3;
  const long long cap = 2LL * c->num_sms, need = (ncell + 255) / 256;
  k_invert_hard<PATH><<<(unsigned)(need < cap ? need : cap), 256, 0, c->stream>>>(
      d, ph, c->d_U, pb, pf, pflag, c->d_geom, c->d_aux, c->d_rare, c->d_nrare, stats, hard, c->d_nhard,
      reinterpret_cast<const MlpPacked*>(c->d_mlp));
  c->launches += 2;
  CK(cudaGetLastError());
  return 0;
}

// The tensor-core record follows the mma.sync record in the context's network buffer.
static inline const MlpTc* mlp_tc_of(const harm_ctx* c) {
  return reinterpret_cast<const MlpTc*>(reinterpret_cast<const char*>(c->d_mlp) + sizeof(MlpPacked));
}
static inline MlpTc* mlp_tc_of(harm_ctx* c) {
  return reinterpret_cast<MlpTc*>(reinterpret_cast<char*>(c->d_mlp) + sizeof(MlpPacked));
}

// Resident blocks per SM of a tensor-core kernel of 256 threads, from its registers and shared
// memory (at most 4 by its shared memory, so its TMEM columns always fit: 4 x 128 = 512),
// after raising its dynamic shared-memory limit, once per device and kernel.
template <typename K>
static int tc_blocks_per_sm(harm_ctx* c, K kernel, std::atomic<unsigned long long>& configured, std::atomic<int>& per_sm) {
  if (c->device < 0 || c->device >= 64) return hb_seterr("tensor-core kernel set-up", cudaErrorInvalidDevice);
  if (!(configured.load(std::memory_order_acquire) & (1ull << c->device))) {
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpTcBlock)));
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, kernel));
    int regs_sm = 0, smem_sm = 0, resv = 0, thr_sm = 0;
    CK(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, c->device));
    CK(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device));
    CK(cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, c->device));
    CK(cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, c->device));
    const int by_regs = regs_sm / (((fa.numRegs + 7) / 8) * 8 * 256);
    const int by_smem = smem_sm / ((int)sizeof(MlpTcBlock) + (int)fa.sharedSizeBytes + resv);
    int n = by_regs < by_smem ? by_regs : by_smem;
    n = n < thr_sm / 256 ? n : thr_sm / 256;
    n = n < 4 ? n : 4;
    per_sm.store(n < 1 ? 1 : n, std::memory_order_relaxed);
    configured.fetch_or(1ull << c->device, std::memory_order_acq_rel);
  }
  return 0;
}

// the common-path inversion with the tensor-core learned start (k_invert_tc)
template <int PATH>
static int launch_invert_tc(harm_ctx* c, const Dims& d, const Phys& ph, const double* pb, double* pf, int8_t* pflag,
                            double* stats) {
  static std::atomic<unsigned long long> configured{0};
  static std::atomic<int> per_sm{1};
  if (int rc = tc_blocks_per_sm(c, k_invert_tc<PATH>, configured, per_sm)) return rc;
  const Tile128 tt = tile128_of(d);
  const long long pairs = ((long long)tt.gx * tt.gy * tt.gz + 1) / 2;
  const long long cap = (long long)per_sm.load(std::memory_order_relaxed) * c->num_sms;
  const unsigned grid = (unsigned)(pairs < cap ? pairs : cap);
  k_invert_tc<PATH><<<grid, 256, sizeof(MlpTcBlock), c->stream>>>(d, ph, c->d_U, pb, pf, pflag, c->d_geom, c->d_aux,
                                                                   c->d_rare, c->d_nrare, stats, tt, mlp_tc_of(c),
                                                                   c->d_status);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

// the learned start of every active cell into wpg with k_mlp_guess_tc
template <int PATH>
static int launch_mlp_guess_tc(harm_ctx* c, const Dims& d) {
  static std::atomic<unsigned long long> configured{0};
  static std::atomic<int> per_sm{1};
  if (int rc = tc_blocks_per_sm(c, k_mlp_guess_tc<PATH>, configured, per_sm)) return rc;
  const Tile128 tt = tile128_of(d);
  const long long pairs = ((long long)tt.gx * tt.gy * tt.gz + 1) / 2;
  const long long cap = (long long)per_sm.load(std::memory_order_relaxed) * c->num_sms;
  const unsigned grid = (unsigned)(pairs < cap ? pairs : cap);
  k_mlp_guess_tc<PATH><<<grid, 256, sizeof(MlpTcBlock), c->stream>>>(d, c->d_U, c->d_geom, c->d_wpg, tt, mlp_tc_of(c),
                                                                      c->d_status);
  c->launches++;
  CK(cudaGetLastError());
  return 0;
}

}  // namespace hb
