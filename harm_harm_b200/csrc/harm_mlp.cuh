// harm_mlp.cuh -- the learned initial guess of the inversion (device side).
//
// A 10 -> 64 -> 64 -> 64 -> 2 network with SiLU activations maps invariants of one cell's
// conserved state and metric to a starting point of Jon's 1-D Newton iteration on W'
// (set_guess_Wp, utoprim_jon.c:890, is the hook it replaces).  Outputs: log(W'/D) and
// log(1 + utsq) = log(gamma^2) (v^2 = utsq/(1+utsq)); the Newton iteration uses the first.
//
// Features, from the alpha-scaled setup quantities of compute_setup_quantities
// (utoprim_jon.c:716) of U/sqrt(-g) and from the metric record (slog(x) = sign(x) log(1+|x|)):
//   0 log D            1 slog(B^2/D)      2 slog(Qt^2/D^2)    3 slog((Q.B)^2/D^3)
//   4 slog(-Q.n'/D)    5 slog(Qt^2/((Q.n')^2 + D^2))
//   6 alpha            7 log sqrt(-g)     8 beta^2/alpha^2    9 g_tt + 1
// Each feature and target is standardised by a mean and a standard deviation of the
// training set (the normalisation record).
//
// Parameters (FP32 master copy, 9154 floats): W1[10][64] b1[64] W2[64][64] b2[64]
// W3[64][64] b3[64] W4[64][2] b4[2], W[in][out].  Inference uses a packed copy: BF16 weights
// in the register-fragment order of mma.sync m16n8k16 (row.col) so that each lane loads
// the B fragments of two adjacent tiles with one 16-byte shared-memory read, FP32 biases and
// the normalisation; the weights and biases of layers 1-3 are halved (see mlp_tanh).
// A warp evaluates its 32 cells as two 16-row tiles; the FP32 accumulator fragment of one
// layer is, after SiLU and conversion to BF16, exactly the A fragment of the next layer,
// so activations never leave registers.
#pragma once
#include <cuda_bf16.h>
#include "harm_invert.cuh"
#include "harm_weno_f32x2.cuh"

namespace hb {

constexpr int MLP_IN = 10, MLP_H = 64, MLP_OUT = 2;
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_IN * MLP_H;     // 640
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;              // 704
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;      // 4800
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;              // 4864
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_H * MLP_H;      // 8960
constexpr int MLP_OFF_W4 = MLP_OFF_B3 + MLP_H;              // 9024
constexpr int MLP_OFF_B4 = MLP_OFF_W4 + MLP_H * MLP_OUT;    // 9152
constexpr int MLP_NPARAMS = MLP_OFF_B4 + MLP_OUT;           // 9154
constexpr int MLP_NNORM = 2 * MLP_IN + 2 * MLP_OUT;         // fmu[10] fsd[10] tmu[2] tsd[2]

// packed inference record: 76 B-fragment tiles (layer 1: 8, layers 2-3: 32 each, layer 4:
// 4) of 32 lanes x 2 words, then biases b1 b2 b3 b4 (+2 pad), the normalisation and the
// start bias
constexpr int MLP_TILES = 8 + 32 + 32 + 4;
constexpr int MLP_TILE_L1 = 0, MLP_TILE_L2 = 8, MLP_TILE_L3 = 40, MLP_TILE_L4 = 72;
constexpr int MLP_NBIAS = 3 * MLP_H + MLP_OUT + 2;
struct MlpPacked {
  uint4 frag[MLP_TILES / 2][32];  // tile pair p, lane l: {tile 2p: b0b1, b2b3; tile 2p+1: b0b1, b2b3}
  float bias[MLP_NBIAS];
  float norm[MLP_NNORM];
  float start_bias;  // added to log(W'/D) before the Newton start (see mlp_wp_guess)
  float pad[3];
};
static_assert(sizeof(MlpPacked) % 16 == 0, "packed record is copied as 16-byte words");

// slog of a ratio formed in FP64 (so that no product of invariants overflows) and taken in
// FP32: the features are FP32 inputs of a BF16 network, so FP32 logarithms lose nothing
__device__ __forceinline__ float mlp_slog(double x) {
  const float xf = (float)fmax(fmin(x, 1e38), -1e38);
  return copysignf(log1pf(fabsf(xf)), xf);
}

// features of one cell from its inversion setup (alpha-scaled quantities) and metric
__device__ __forceinline__ void mlp_features(const InvC& c, const Geo<double>& g, float* f) {
  const double D = (c.D > 1e-300) ? c.D : 1e-300;
  const double iD = 1.0 / D;
  f[0] = logf(fmaxf((float)fmin(D, 1e38), 1e-38f));
  f[1] = mlp_slog(c.Bsq * iD);
  f[2] = mlp_slog(c.Qtsq * iD * iD);
  f[3] = mlp_slog(c.QdotBsq * iD * iD * iD);
  f[4] = mlp_slog(-c.Qdotnp * iD);
  f[5] = mlp_slog(c.Qtsq / (c.Qdotnp * c.Qdotnp + D * D));
  f[6] = (float)g.alpha;
  f[7] = logf(fmaxf((float)fmin(fabs(g.gdet), 1e38), 1e-38f));
  f[8] = (float)g.betasqoalphasq;
  f[9] = (float)g.gcovpert_tt;
}

// targets of a converged inversion: log(W'/D), log(1 + utsq)
__device__ __forceinline__ void mlp_targets(double Wp, const InvC& c, float* t) {
  const double D = (c.D > 1e-300) ? c.D : 1e-300;
  const double r = Wp / D;
  t[0] = (float)log(r > 1e-300 ? r : 1e-300);
  const double utsq = utsq_calc(Wp + c.D, c);
  t[1] = (float)log1p(utsq > 0.0 ? utsq : 0.0);
}

// SiLU of the inference.  x sigmoid(x) = h + h tanh(h) with h = x/2; the packed records hold
// the weights and biases of layers 1-3 halved (exact in BF16 and FP32: a power of two), so
// the accumulators are h itself.  Hardware tanh approximation (one special-function operation;
// its error, about 2^-11, is below the BF16 rounding the activation receives next), then one
// packed FP32x2 FMA for two activations.
__device__ __forceinline__ float mlp_tanh(float h) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(h));
  return t;
}
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half), .y = hi
  return *reinterpret_cast<uint32_t*>(&v);
}

// two activations from their halves h, as BF16x2 (the first in the low half)
__device__ __forceinline__ uint32_t mlp_silu2_bf16(F2 h) {
  float h0, h1;
  f2split(h, h0, h1);
  float s0, s1;
  f2split(ffma2(h, f2(mlp_tanh(h0), mlp_tanh(h1)), h), s0, s1);
  return pack_bf16x2(s0, s1);
}

__device__ __forceinline__ void mma_bf16_16816(float* c, const uint32_t* a, uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// Per-warp scratch of the inference: the BF16 input rows (32 cells x 12 words; 8 used,
// the stride keeps the fragment reads free of bank conflicts) and the outputs.
struct MlpWarpScratch {
  uint32_t x[32 * 12];
  float y[32 * 2];
};

// SiLU of two accumulator tiles (n-tiles 2q, 2q+1) as the A fragment of k-tile q
__device__ __forceinline__ void mlp_act_to_a(const float* c0, const float* c1, uint32_t* a) {
  a[0] = mlp_silu2_bf16(f2(c0[0], c0[1]));
  a[1] = mlp_silu2_bf16(f2(c0[2], c0[3]));
  a[2] = mlp_silu2_bf16(f2(c1[0], c1[1]));
  a[3] = mlp_silu2_bf16(f2(c1[2], c1[3]));
}

// Evaluate the network for the 32 cells of this warp.  All 32 lanes must call it (lanes
// without a cell pass valid = false).  f: this lane's 10 raw features; out: this lane's
// de-standardised outputs.
__device__ __forceinline__ void mlp_warp_eval(const MlpPacked& m, MlpWarpScratch& ws, const float* f, bool valid,
                                              float* out) {
  const int lane = threadIdx.x & 31, q = lane & 3, grp = lane >> 2;
  {
    float x[12];
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) x[i] = valid ? (f[i] - m.norm[i]) / m.norm[MLP_IN + i] : 0.0f;
    x[10] = 0.0f;
    x[11] = 0.0f;
    uint32_t* row = ws.x + lane * 12;
#pragma unroll
    for (int w = 0; w < 6; w++) row[w] = pack_bf16x2(x[2 * w], x[2 * w + 1]);
    row[6] = 0u;
    row[7] = 0u;
  }
  __syncwarp();
  const float* b1 = m.bias;
  const float* b2 = m.bias + MLP_H;
  const float* b3 = m.bias + 2 * MLP_H;
  const float* b4 = m.bias + 3 * MLP_H;
#pragma unroll 1
  for (int mt = 0; mt < 2; mt++) {
    const int r0 = mt * 16 + grp, r1 = r0 + 8;
    uint32_t a[4][4];
    float acc[8][4];
    {
      uint32_t a1[4] = {ws.x[r0 * 12 + q], ws.x[r1 * 12 + q], ws.x[r0 * 12 + 4 + q], ws.x[r1 * 12 + 4 + q]};
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        const float bl = b1[nt * 8 + 2 * q], bh = b1[nt * 8 + 2 * q + 1];
        acc[nt][0] = bl; acc[nt][1] = bh; acc[nt][2] = bl; acc[nt][3] = bh;
      }
#pragma unroll
      for (int np = 0; np < 4; np++) {
        const uint4 bb = m.frag[MLP_TILE_L1 / 2 + np][lane];
        mma_bf16_16816(acc[2 * np], a1, make_uint2(bb.x, bb.y));
        mma_bf16_16816(acc[2 * np + 1], a1, make_uint2(bb.z, bb.w));
      }
    }
#pragma unroll
    for (int kt = 0; kt < 4; kt++) mlp_act_to_a(acc[2 * kt], acc[2 * kt + 1], a[kt]);
#pragma unroll
    for (int layer = 0; layer < 2; layer++) {
      const float* bb = layer ? b3 : b2;
      const int base = layer ? MLP_TILE_L3 : MLP_TILE_L2;
#pragma unroll
      for (int nt = 0; nt < 8; nt++) {
        const float bl = bb[nt * 8 + 2 * q], bh = bb[nt * 8 + 2 * q + 1];
        acc[nt][0] = bl; acc[nt][1] = bh; acc[nt][2] = bl; acc[nt][3] = bh;
      }
#pragma unroll
      for (int kt = 0; kt < 4; kt++)
#pragma unroll
        for (int np = 0; np < 4; np++) {
          const uint4 bb = m.frag[(base + kt * 8) / 2 + np][lane];
          mma_bf16_16816(acc[2 * np], a[kt], make_uint2(bb.x, bb.y));
          mma_bf16_16816(acc[2 * np + 1], a[kt], make_uint2(bb.z, bb.w));
        }
#pragma unroll
      for (int kt = 0; kt < 4; kt++) mlp_act_to_a(acc[2 * kt], acc[2 * kt + 1], a[kt]);
    }
    float o[4];
    o[0] = (q == 0) ? b4[0] : 0.0f;
    o[1] = (q == 0) ? b4[1] : 0.0f;
    o[2] = o[0];
    o[3] = o[1];
#pragma unroll
    for (int kp = 0; kp < 2; kp++) {
      const uint4 bb = m.frag[MLP_TILE_L4 / 2 + kp][lane];
      mma_bf16_16816(o, a[2 * kp], make_uint2(bb.x, bb.y));
      mma_bf16_16816(o, a[2 * kp + 1], make_uint2(bb.z, bb.w));
    }
    if (q == 0) {
      ws.y[r0 * 2 + 0] = o[0];
      ws.y[r0 * 2 + 1] = o[1];
      ws.y[r1 * 2 + 0] = o[2];
      ws.y[r1 * 2 + 1] = o[3];
    }
  }
  __syncwarp();
  const float* nrm = m.norm + 2 * MLP_IN;
  out[0] = ws.y[lane * 2 + 0] * nrm[MLP_OUT + 0] + nrm[0];
  out[1] = ws.y[lane * 2 + 1] * nrm[MLP_OUT + 1] + nrm[1];
  __syncwarp();
}

// block-cooperative copy of the packed record into shared memory
__device__ __forceinline__ void mlp_load_packed(MlpPacked& dst, const MlpPacked* __restrict__ src) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(&dst);
  for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) d[i] = __ldg(s + i);
}

// Starting W' from the network's first output, raised by the record's start_bias in log
// space: Newton on E'(W') converges from above the root without verify_Wlast's corrections
// (a start below the root can give v^2 > 1, which that check answers by raising W' tenfold),
// so a start a few network errors above the prediction is the robust side.
// NaN/inf/non-positive: the previous-state W'.
__device__ __forceinline__ double mlp_wp_guess(float y0, float start_bias, const JonSetup& s) {
  double wp = s.c.D * exp((double)y0 + (double)start_bias);
  return (wp > 0.0 && isfinite(wp)) ? wp : s.Wp_prev;
}

}  // namespace hb
