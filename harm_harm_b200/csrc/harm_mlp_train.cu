// harm_mlp_train.cu -- training and inference plumbing of the learned inversion guess.
//
// Training runs in FP32 with hand-written kernels:
//   k_mlp_grad   forward and backward pass of the 10-64-64-64-2 SiLU network over a
//                minibatch; each block owns a slice of the samples, keeps the parameters,
//                activations and its gradient accumulators in shared memory (208 KB) and
//                writes one partial gradient, so the reduction order is fixed
//                (deterministic gradients);
//   k_mlp_adam   sums the partial gradients in block order and applies Adam;
//   k_mlp_norm   feature/target means and standard deviations (one block, FP64 sums);
//   k_mlp_init   Glorot-uniform weights, zero biases, from a counter-based hash.
// Loss: L = 1/(2n) sum_samples sum_outputs (y - t~)^2 over the standardised targets t~.
// Inference: k_mlp_pack writes the BF16 fragment-ordered record of harm_mlp.cuh;
// k_mlp_predict evaluates it on the tensor cores (mma.sync m16n8k16, FP32 accumulation),
// the same device function the inversion kernels call.
#include <algorithm>
#include <vector>
#include "harm_common.cuh"
#include "harm_mlp.cuh"
#include "harm_mlp_tc.cuh"

int hb_setmsg(const char* msg, int code);

namespace {

constexpr int TS = 64;           // samples per chunk
constexpr int NPP = 9156;        // parameters padded to a multiple of 4
constexpr int TR_GRID = 128;     // blocks of one training step
constexpr size_t TR_SMEM = (size_t)(2 * NPP + TS * MLP_IN + 6 * TS * MLP_H + TS * 2 + 2 * TS * MLP_H + TS * 2 + 8) * 4;
static_assert(MLP_NPARAMS <= NPP, "padding");

__device__ __forceinline__ uint64_t smix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Z = Hin W + b over a chunk (64 samples x 64 outputs); Hout = silu(Z)
__device__ __forceinline__ void dense64(const float* Hin, const float* W, const float* b, float* Z, float* Hout) {
  for (int e = threadIdx.x; e < TS * MLP_H; e += blockDim.x) {
    const int s = e >> 6, o = e & 63;
    float z = b[o];
    const float* h = Hin + s * MLP_H;
#pragma unroll 8
    for (int k = 0; k < MLP_H; k++) z += h[k] * W[k * MLP_H + o];
    Z[e] = z;
    Hout[e] = silu_f(z);
  }
}

// gW[i][o] += sum_s Hin[s][i] D[s][o];  gb[o] += sum_s D[s][o]
__device__ __forceinline__ void wgrad64(const float* Hin, int nin, const float* D, float* gW, float* gb) {
  for (int e = threadIdx.x; e < nin * MLP_H; e += blockDim.x) {
    const int i = e >> 6, o = e & 63;
    float a = 0.0f;
#pragma unroll 8
    for (int s = 0; s < TS; s++) a += Hin[s * nin + i] * D[s * MLP_H + o];
    gW[e] += a;
  }
  for (int o = threadIdx.x; o < MLP_H; o += blockDim.x) {
    float a = 0.0f;
    for (int s = 0; s < TS; s++) a += D[s * MLP_H + o];
    gb[o] += a;
  }
}

// Dout[s][i] = silu'(Zprev[s][i]) * sum_o Din[s][o] W[i][o]  (o rotated by i: no bank conflicts)
__device__ __forceinline__ void bwd64(const float* Din, const float* W, const float* Zprev, float* Dout) {
  for (int e = threadIdx.x; e < TS * MLP_H; e += blockDim.x) {
    const int s = e >> 6, i = e & 63;
    const float* dz = Din + s * MLP_H;
    const float* w = W + i * MLP_H;
    float a = 0.0f;
#pragma unroll 8
    for (int oo = 0; oo < MLP_H; oo++) {
      const int o = (oo + i) & 63;
      a += dz[o] * w[o];
    }
    Dout[e] = a * dsilu_f(Zprev[e]);
  }
}

__global__ void __launch_bounds__(256, 1) k_mlp_grad(size_t ndata, const float* __restrict__ feat,
                                                     const float* __restrict__ targ, const float* __restrict__ norm,
                                                     const float* __restrict__ params, long long nbatch,
                                                     uint64_t seed, long long step, float inv_n,
                                                     float* __restrict__ partial, double* __restrict__ partial_loss) {
  extern __shared__ __align__(16) float sm[];
  float* P = sm;
  float* G = P + NPP;
  float* X = G + NPP;
  float* Z1 = X + TS * MLP_IN;
  float* Z2 = Z1 + TS * MLP_H;
  float* Z3 = Z2 + TS * MLP_H;
  float* H1 = Z3 + TS * MLP_H;
  float* H2 = H1 + TS * MLP_H;
  float* H3 = H2 + TS * MLP_H;
  float* DY = H3 + TS * MLP_H;
  float* DA = DY + TS * 2;
  float* DB = DA + TS * MLP_H;
  float* T = DB + TS * MLP_H;
  float* red = T + TS * 2;
  const int tid = threadIdx.x;
  for (int i = tid; i < NPP; i += blockDim.x) {
    P[i] = (i < MLP_NPARAMS) ? params[i] : 0.0f;
    G[i] = 0.0f;
  }
  const long long per = (nbatch + gridDim.x - 1) / gridDim.x;
  const long long s0 = (long long)blockIdx.x * per, s1 = min(nbatch, s0 + per);
  float lacc = 0.0f;
  for (long long c0 = s0; c0 < s1; c0 += TS) {
    const int nc = (int)min((long long)TS, s1 - c0);
    __syncthreads();
    for (int e = tid; e < TS * 12; e += blockDim.x) {
      const int s = e / 12, col = e % 12;
      float v = 0.0f;
      if (s < nc) {
        const long long j = c0 + s;
        const size_t idx = seed ? (size_t)(smix(seed ^ smix((uint64_t)(step * nbatch + j))) % ndata) : (size_t)j;
        if (col < MLP_IN) v = (feat[idx * MLP_IN + col] - norm[col]) / norm[MLP_IN + col];
        else v = (targ[idx * MLP_OUT + col - MLP_IN] - norm[2 * MLP_IN + col - MLP_IN]) / norm[2 * MLP_IN + 2 + col - MLP_IN];
      }
      if (col < MLP_IN) X[s * MLP_IN + col] = v;
      else T[s * 2 + col - MLP_IN] = v;
    }
    __syncthreads();
    // layer 1
    for (int e = tid; e < TS * MLP_H; e += blockDim.x) {
      const int s = e >> 6, o = e & 63;
      float z = P[MLP_OFF_B1 + o];
#pragma unroll
      for (int i = 0; i < MLP_IN; i++) z += X[s * MLP_IN + i] * P[MLP_OFF_W1 + i * MLP_H + o];
      Z1[e] = z;
      H1[e] = silu_f(z);
    }
    __syncthreads();
    dense64(H1, P + MLP_OFF_W2, P + MLP_OFF_B2, Z2, H2);
    __syncthreads();
    dense64(H2, P + MLP_OFF_W3, P + MLP_OFF_B3, Z3, H3);
    __syncthreads();
    // output and its error
    if (tid < TS * 2) {
      const int s = tid >> 1, o = tid & 1;
      float y = P[MLP_OFF_B4 + o];
#pragma unroll 8
      for (int k = 0; k < MLP_H; k++) y += H3[s * MLP_H + k] * P[MLP_OFF_W4 + k * 2 + o];
      float dy = 0.0f;
      if (s < nc) {
        const float r = y - T[s * 2 + o];
        lacc += 0.5f * r * r;
        dy = r * inv_n;
      }
      DY[tid] = dy;
    }
    __syncthreads();
    if (tid < MLP_H * 2) {
      const int k = tid >> 1, o = tid & 1;
      float a = 0.0f;
      for (int s = 0; s < TS; s++) a += H3[s * MLP_H + k] * DY[s * 2 + o];
      G[MLP_OFF_W4 + tid] += a;
    }
    if (tid < 2) {
      float a = 0.0f;
      for (int s = 0; s < TS; s++) a += DY[s * 2 + tid];
      G[MLP_OFF_B4 + tid] += a;
    }
    for (int e = tid; e < TS * MLP_H; e += blockDim.x) {
      const int s = e >> 6, k = e & 63;
      const float dh = DY[s * 2] * P[MLP_OFF_W4 + k * 2] + DY[s * 2 + 1] * P[MLP_OFF_W4 + k * 2 + 1];
      DA[e] = dh * dsilu_f(Z3[e]);
    }
    __syncthreads();
    wgrad64(H2, MLP_H, DA, G + MLP_OFF_W3, G + MLP_OFF_B3);
    bwd64(DA, P + MLP_OFF_W3, Z2, DB);
    __syncthreads();
    wgrad64(H1, MLP_H, DB, G + MLP_OFF_W2, G + MLP_OFF_B2);
    bwd64(DB, P + MLP_OFF_W2, Z1, DA);
    __syncthreads();
    wgrad64(X, MLP_IN, DA, G + MLP_OFF_W1, G + MLP_OFF_B1);
  }
  __syncthreads();
  for (int i = tid; i < MLP_NPARAMS; i += blockDim.x) partial[(size_t)blockIdx.x * MLP_NPARAMS + i] = G[i];
  // block loss in a fixed order
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lacc += __shfl_xor_sync(0xffffffffu, lacc, o);
  if ((tid & 31) == 0) red[tid >> 5] = lacc;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    partial_loss[blockIdx.x] = s;
  }
}

// sum of the partial gradients (block order), then Adam when lr > 0
__global__ void k_mlp_adam(int nb, const float* __restrict__ partial, const double* __restrict__ partial_loss,
                           float* __restrict__ params, float* __restrict__ m, float* __restrict__ v, float lr,
                           float b1, float b2, float eps, float bc1, float bc2, float inv_n,
                           float* __restrict__ grad_out, double* __restrict__ loss_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < MLP_NPARAMS) {
    float g = 0.0f;
    for (int b = 0; b < nb; b++) g += partial[(size_t)b * MLP_NPARAMS + p];
    if (grad_out) grad_out[p] = g;
    if (lr > 0.0f) {
      const float mm = b1 * m[p] + (1.0f - b1) * g;
      const float vv = b2 * v[p] + (1.0f - b2) * g * g;
      m[p] = mm;
      v[p] = vv;
      params[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
    }
  }
  if (p == 0 && loss_out) {
    double s = 0.0;
    for (int b = 0; b < nb; b++) s += partial_loss[b];
    *loss_out = s * (double)inv_n;
  }
}

__global__ void k_mlp_norm(size_t n, const float* __restrict__ feat, const float* __restrict__ targ,
                           float* __restrict__ norm) {
  __shared__ double s1[MLP_IN + MLP_OUT][32], s2[MLP_IN + MLP_OUT][32];
  double a1[MLP_IN + MLP_OUT], a2[MLP_IN + MLP_OUT];
  for (int c = 0; c < MLP_IN + MLP_OUT; c++) { a1[c] = 0.0; a2[c] = 0.0; }
  for (size_t t = threadIdx.x; t < n; t += blockDim.x) {
    for (int c = 0; c < MLP_IN; c++) {
      double x = feat[t * MLP_IN + c];
      a1[c] += x; a2[c] += x * x;
    }
    for (int c = 0; c < MLP_OUT; c++) {
      double x = targ[t * MLP_OUT + c];
      a1[MLP_IN + c] += x; a2[MLP_IN + c] += x * x;
    }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int c = 0; c < MLP_IN + MLP_OUT; c++) {
    double x = a1[c], y = a2[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      y += __shfl_xor_sync(0xffffffffu, y, o);
    }
    if (lane == 0) { s1[c][w] = x; s2[c][w] = y; }
  }
  __syncthreads();
  if (threadIdx.x < MLP_IN + MLP_OUT) {
    const int c = threadIdx.x;
    double x = 0.0, y = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) { x += s1[c][q]; y += s2[c][q]; }
    const double mean = x / (double)n, var = fmax(y / (double)n - mean * mean, 0.0);
    double sd = sqrt(var);
    if (!(sd > 1e-6)) sd = 1.0;
    if (c < MLP_IN) { norm[c] = (float)mean; norm[MLP_IN + c] = (float)sd; }
    else { norm[2 * MLP_IN + c - MLP_IN] = (float)mean; norm[2 * MLP_IN + MLP_OUT + c - MLP_IN] = (float)sd; }
  }
}

__global__ void k_mlp_init(uint64_t seed, float* __restrict__ params) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= MLP_NPARAMS) return;
  int fin = 0, fout = 0;
  if (p < MLP_OFF_B1) { fin = MLP_IN; fout = MLP_H; }
  else if (p >= MLP_OFF_W2 && p < MLP_OFF_B2) { fin = MLP_H; fout = MLP_H; }
  else if (p >= MLP_OFF_W3 && p < MLP_OFF_B3) { fin = MLP_H; fout = MLP_H; }
  else if (p >= MLP_OFF_W4 && p < MLP_OFF_B4) { fin = MLP_H; fout = MLP_OUT; }
  if (fin == 0) { params[p] = 0.0f; return; }
  const double u = (double)(smix(seed ^ smix((uint64_t)p)) >> 11) * (1.0 / 9007199254740992.0);
  const double a = sqrt(6.0 / (double)(fin + fout));
  params[p] = (float)((2.0 * u - 1.0) * a);
}

// BF16 fragments (mma.sync m16n8k16 .col B operand), biases, normalisation, start bias
__global__ void k_mlp_pack(const float* __restrict__ params, const float* __restrict__ norm, float start_bias,
                           MlpPacked* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < MLP_TILES * 32) {
    const int tile = t >> 5, lane = t & 31;
    int woff, K, N, kt, nt;
    if (tile < MLP_TILE_L2) { woff = MLP_OFF_W1; K = MLP_IN; N = MLP_H; kt = 0; nt = tile; }
    else if (tile < MLP_TILE_L3) { woff = MLP_OFF_W2; K = MLP_H; N = MLP_H; kt = (tile - MLP_TILE_L2) >> 3; nt = (tile - MLP_TILE_L2) & 7; }
    else if (tile < MLP_TILE_L4) { woff = MLP_OFF_W3; K = MLP_H; N = MLP_H; kt = (tile - MLP_TILE_L3) >> 3; nt = (tile - MLP_TILE_L3) & 7; }
    else { woff = MLP_OFF_W4; K = MLP_H; N = MLP_OUT; kt = tile - MLP_TILE_L4; nt = 0; }
    const int k0 = kt * 16 + 2 * (lane & 3), n = nt * 8 + (lane >> 2);
    const float scale = (tile < MLP_TILE_L4) ? 0.5f : 1.0f;  // layers 1-3 halved (mlp_tanh)
    auto W = [&](int k) -> float { return (k < K && n < N) ? scale * params[woff + k * N + n] : 0.0f; };
    uint32_t* f = reinterpret_cast<uint32_t*>(&out->frag[tile >> 1][lane]) + 2 * (tile & 1);
    f[0] = pack_bf16x2(W(k0), W(k0 + 1));
    f[1] = pack_bf16x2(W(k0 + 8), W(k0 + 9));
  }
  if (t < MLP_NBIAS) {
    float b = 0.0f;
    if (t < MLP_H) b = 0.5f * params[MLP_OFF_B1 + t];
    else if (t < 2 * MLP_H) b = 0.5f * params[MLP_OFF_B2 + t - MLP_H];
    else if (t < 3 * MLP_H) b = 0.5f * params[MLP_OFF_B3 + t - 2 * MLP_H];
    else if (t < 3 * MLP_H + MLP_OUT) b = params[MLP_OFF_B4 + t - 3 * MLP_H];
    out->bias[t] = b;
  }
  if (t < MLP_NNORM) out->norm[t] = norm[t];
  if (t == 0) {
    out->start_bias = start_bias;
    out->pad[0] = out->pad[1] = out->pad[2] = 0.0f;
  }
}

// BF16 B operands in the tensor-core canonical layout of harm_mlp_tc.cuh (one 16-byte chunk of
// 8 K-consecutive weights per thread), biases, normalisation, start bias
__global__ void k_mlp_pack_tc(const float* __restrict__ params, const float* __restrict__ norm, float start_bias,
                              MlpTc* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < TC_WBYTES / 16) {
    const int off = t * 16;
    int base, kc, woff, K, N;
    if (off < TC_W2) { base = TC_W1; kc = 2; woff = MLP_OFF_W1; K = MLP_IN; N = MLP_H; }
    else if (off < TC_W3) { base = TC_W2; kc = 8; woff = MLP_OFF_W2; K = MLP_H; N = MLP_H; }
    else if (off < TC_W4) { base = TC_W3; kc = 8; woff = MLP_OFF_W3; K = MLP_H; N = MLP_H; }
    else { base = TC_W4; kc = 8; woff = MLP_OFF_W4; K = MLP_H; N = MLP_OUT; }
    const int rel = off - base, cm = rel >> 7;
    const int n = (cm / kc) * 8 + ((rel & 127) >> 4), k0 = (cm % kc) * 8;  // tc_off(n, k0, kc) == rel
    const float scale = (base < TC_W4) ? 0.5f : 1.0f;  // layers 1-3 halved (mlp_tanh)
    auto W = [&](int k) -> float { return (k < K && n < N) ? scale * params[woff + k * N + n] : 0.0f; };
    uint4 v;
    v.x = pack_bf16x2(W(k0), W(k0 + 1));
    v.y = pack_bf16x2(W(k0 + 2), W(k0 + 3));
    v.z = pack_bf16x2(W(k0 + 4), W(k0 + 5));
    v.w = pack_bf16x2(W(k0 + 6), W(k0 + 7));
    out->w[t] = v;
  }
  if (t < MLP_NBIAS) {
    float b = 0.0f;
    if (t < MLP_H) b = 0.5f * params[MLP_OFF_B1 + t];
    else if (t < 2 * MLP_H) b = 0.5f * params[MLP_OFF_B2 + t - MLP_H];
    else if (t < 3 * MLP_H) b = 0.5f * params[MLP_OFF_B3 + t - 2 * MLP_H];
    else if (t < 3 * MLP_H + MLP_OUT) b = params[MLP_OFF_B4 + t - 3 * MLP_H];
    out->bias[t] = b;
  }
  if (t < MLP_NNORM) out->norm[t] = norm[t];
  if (t == 0) {
    out->start_bias = start_bias;
    out->pad[0] = out->pad[1] = out->pad[2] = 0.0f;
  }
}

__global__ void __launch_bounds__(256) k_mlp_predict(size_t n, const float* __restrict__ feat,
                                                     const MlpPacked* __restrict__ mlp, float* __restrict__ out) {
  __shared__ MlpPacked sm;
  __shared__ MlpWarpScratch ws[8];
  mlp_load_packed(sm, mlp);
  __syncthreads();
  for (size_t base = (size_t)blockIdx.x * 256; base < n; base += (size_t)gridDim.x * 256) {
    const size_t t = base + threadIdx.x;
    const bool valid = t < n;
    float f[MLP_IN];
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) f[i] = valid ? feat[t * MLP_IN + i] : 0.0f;
    float y[MLP_OUT];
    mlp_warp_eval(sm, ws[threadIdx.x >> 5], f, valid, y);
    if (valid) {
      out[t * MLP_OUT + 0] = y[0];
      out[t * MLP_OUT + 1] = y[1];
    }
  }
}

int ensure_train_scratch(harm_ctx* c) {
  if (!c->d_mlp_adam) {
    CK(cudaMalloc(&c->d_mlp_adam, 2 * (size_t)MLP_NPARAMS * sizeof(float)));
  }
  if (!c->d_mlp_work) {
    // partial gradients of up to TR_GRID blocks, their partial losses (doubles) and the loss
    c->mlp_work_n = (size_t)TR_GRID * MLP_NPARAMS + 2 * TR_GRID + 4;
    CK(cudaMalloc(&c->d_mlp_work, c->mlp_work_n * sizeof(float)));
  }
  static std::atomic<unsigned long long> raised{0};
  CK(raise_smem_limit_once(raised, (const void*)k_mlp_grad, (int)TR_SMEM));
  return 0;
}

double* partial_loss_of(harm_ctx* c) {
  return reinterpret_cast<double*>(c->d_mlp_work + (size_t)TR_GRID * MLP_NPARAMS + 2);  // 8-byte aligned
}

}  // namespace

extern "C" int harm_b200_mlp_init(harm_ctx* c, uint64_t seed, float* d_params) {
  if (!c || !d_params) return hb_setmsg("null argument", 1);
  k_mlp_init<<<nblk(MLP_NPARAMS), 256, 0, c->stream>>>(seed, d_params);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int harm_b200_mlp_norm(harm_ctx* c, size_t n, const float* d_feat, const float* d_targ, float* d_norm) {
  if (!c || !d_feat || !d_targ || !d_norm) return hb_setmsg("null argument", 1);
  if (n == 0) return hb_setmsg("no samples", 2);
  k_mlp_norm<<<1, 1024, 0, c->stream>>>(n, d_feat, d_targ, d_norm);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

extern "C" int harm_b200_mlp_loss_grad(harm_ctx* c, size_t n, const float* d_feat, const float* d_targ,
                                       const float* d_params, const float* d_norm, double* loss, float* d_grad) {
  if (!c || !d_feat || !d_targ || !d_params || !d_norm || !d_grad) return hb_setmsg("null argument", 1);
  if (n == 0) return hb_setmsg("no samples", 2);
  if (ensure_train_scratch(c)) return 1;
  const int nb = (int)std::min<size_t>((n + TS - 1) / TS, (size_t)TR_GRID);
  float* partial = c->d_mlp_work;
  double* ploss = partial_loss_of(c);
  double* dloss = ploss + TR_GRID;
  const float inv_n = (float)(1.0 / (double)n);
  k_mlp_grad<<<nb, 256, TR_SMEM, c->stream>>>(n, d_feat, d_targ, d_norm, d_params, (long long)n, 0ull, 0ll, inv_n,
                                              partial, ploss);
  k_mlp_adam<<<nblk(MLP_NPARAMS), 256, 0, c->stream>>>(nb, partial, ploss, nullptr, nullptr, nullptr, 0.0f, 0.f, 0.f,
                                                       0.f, 1.f, 1.f, inv_n, d_grad, dloss);
  c->launches += 2;
  CK(cudaGetLastError());
  double h = 0.0;
  CK(cudaMemcpyAsync(&h, dloss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (loss) *loss = h;
  return 0;
}

extern "C" int harm_b200_mlp_train(harm_ctx* c, size_t n, const float* d_feat, const float* d_targ,
                                   const float* d_norm, float* d_params, int steps, int batch, float lr,
                                   uint64_t seed, float* loss_hist) {
  if (!c || !d_feat || !d_targ || !d_norm || !d_params) return hb_setmsg("null argument", 1);
  if (n == 0 || steps < 1 || batch < 1) return hb_setmsg("need n, steps and batch >= 1", 2);
  if (seed == 0) seed = 0x5eedull;
  if (ensure_train_scratch(c)) return 1;
  float* m = c->d_mlp_adam;
  float* v = m + MLP_NPARAMS;
  CK(cudaMemsetAsync(m, 0, 2 * (size_t)MLP_NPARAMS * sizeof(float), c->stream));
  float* partial = c->d_mlp_work;
  double* ploss = partial_loss_of(c);
  double* dloss = ploss + TR_GRID;
  std::vector<double> hist;
  double* d_hist = nullptr;
  if (loss_hist) {
    CK(cudaMalloc(&d_hist, (size_t)steps * sizeof(double)));
  }
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const int nb = (int)std::min<long long>(((long long)batch + TS - 1) / TS, (long long)TR_GRID);
  const float inv_n = (float)(1.0 / (double)batch);
  double p1 = 1.0, p2 = 1.0;
  for (int s = 0; s < steps; s++) {
    // cosine decay to lr/100
    const double frac = (double)s / (double)steps;
    const float lr_s = (float)(lr * (0.01 + 0.99 * 0.5 * (1.0 + cos(3.141592653589793 * frac))));
    p1 *= b1;
    p2 *= b2;
    k_mlp_grad<<<nb, 256, TR_SMEM, c->stream>>>(n, d_feat, d_targ, d_norm, d_params, (long long)batch, seed,
                                                (long long)s, inv_n, partial, ploss);
    k_mlp_adam<<<nblk(MLP_NPARAMS), 256, 0, c->stream>>>(nb, partial, ploss, d_params, m, v, lr_s, b1, b2, eps,
                                                         (float)(1.0 - p1), (float)(1.0 - p2), inv_n, nullptr,
                                                         d_hist ? d_hist + s : dloss);
    c->launches += 2;
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && d_hist) {
    hist.resize(steps);
    e = cudaMemcpyAsync(hist.data(), d_hist, (size_t)steps * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (d_hist) cudaFree(d_hist);
  if (e != cudaSuccess) return hb_seterr("mlp training", e);
  if (loss_hist)
    for (int s = 0; s < steps; s++) loss_hist[s] = (float)hist[s];
  return 0;
}

extern "C" int harm_b200_mlp_set(harm_ctx* c, const float* d_params, const float* d_norm, double start_bias) {
  if (!c || !d_params || !d_norm) return hb_setmsg("null argument", 1);
  if (!c->d_mlp) {
    CK(cudaMalloc(&c->d_mlp, sizeof(MlpPacked) + sizeof(MlpTc)));
  }
  if (!c->d_wpg) {
    CK(cudaMalloc(&c->d_wpg, (size_t)c->g.n1 * c->g.n2 * c->g.n3 * sizeof(double)));
  }
  k_mlp_pack<<<nblk(MLP_TILES * 32), 256, 0, c->stream>>>(d_params, d_norm, (float)start_bias,
                                                         reinterpret_cast<MlpPacked*>(c->d_mlp));
  k_mlp_pack_tc<<<nblk(TC_WBYTES / 16), 256, 0, c->stream>>>(d_params, d_norm, (float)start_bias, mlp_tc_of(c));
  c->launches += 2;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  c->mlp_step = 1;  // a packed network is present
  return 0;
}

// Network outputs for n feature rows (the tensor-core counterpart of k_mlp_predict).
__global__ void __launch_bounds__(256) k_mlp_predict_tc(size_t n, const float* __restrict__ feat,
                                                        const MlpTc* __restrict__ mlp, float* __restrict__ out,
                                                        unsigned int* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char tc_smem[];
  MlpTcBlock& B = *reinterpret_cast<MlpTcBlock*>(tc_smem);
  mlp_tc_begin(B, mlp);
  const int wg = threadIdx.x >> 7, r = threadIdx.x & 127;
  const long long ntiles = (long long)((n + 127) / 128);
  TcState st = {0u, false};
  for (long long tile = 2ll * blockIdx.x + wg; tile < ntiles; tile += 2ll * gridDim.x) {
    const size_t t = (size_t)tile * 128 + r;
    const bool valid = t < n;
    float f[MLP_IN], x[MLP_IN];
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) f[i] = valid ? feat[t * MLP_IN + i] : 0.0f;
    mlp_tc_standardise(B.net, f, valid, x);
    float y[MLP_OUT];
    if (!mlp_tc_eval(B, x, st, status, y)) break;
    if (valid) {
      out[t * MLP_OUT + 0] = y[0];
      out[t * MLP_OUT + 1] = y[1];
    }
  }
  mlp_tc_end(B, st);
}

extern "C" int harm_b200_mlp_predict(harm_ctx* c, size_t n, const float* d_feat, float* d_out) {
  if (!c || !d_feat || !d_out) return hb_setmsg("null argument", 1);
  if (!c->d_mlp || !c->mlp_step) return hb_setmsg("no network set (harm_b200_mlp_set)", 3);
  if (n == 0) return 0;
  if (c->mlp_tc == 1 || c->mlp_tc == 2) {  // the tcgen05 engines: their network kernel
    static std::atomic<unsigned long long> configured{0};
    static std::atomic<int> per_sm{1};
    if (int rc = tc_blocks_per_sm(c, k_mlp_predict_tc, configured, per_sm)) return rc;
    const size_t pairs = (n + 255) / 256;
    const unsigned int nb = (unsigned int)std::min<size_t>(pairs, (size_t)per_sm.load() * c->num_sms);
    k_mlp_predict_tc<<<nb, 256, sizeof(MlpTcBlock), c->stream>>>(n, d_feat, mlp_tc_of(c), d_out, c->d_status);
  } else {
    const unsigned int nb = (unsigned int)std::min<size_t>((n + 255) / 256, (size_t)4 * c->num_sms);
    k_mlp_predict<<<nb, 256, 0, c->stream>>>(n, d_feat, reinterpret_cast<const MlpPacked*>(c->d_mlp), d_out);
  }
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  unsigned int st = 0;
  CK(cudaMemcpy(&st, c->d_status, sizeof(st), cudaMemcpyDeviceToHost));
  if (st) {
    CK(cudaMemset(c->d_status, 0, sizeof(st)));
    return hb_setmsg("a tensor-core MMA of the network did not complete", 5);
  }
  return 0;
}
