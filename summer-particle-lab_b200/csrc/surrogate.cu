// Learned return map: a small MLP (8 -> 64 -> 64 -> 7, ReLU) that stands in for the J2 /
// thermal-J2 radial return per particle, trained on the GPU from samples the exact map generates.
//
// What it maps. From the trial Hencky strain L = log V of F_trial (Voigt order xx, yy, zz,
// sqrt2 xy, sqrt2 xz, sqrt2 yz), the temperature T and the plastic strain ep, the network sees
// (8 inputs) the unit direction n of dev L, (T - T_lo) / T_span and ep / ep_scale, and predicts
// (7 outputs) the return in the units of the elastic predictor: the correction to the trial
// Kirchhoff stress (tau - tau_trial) / (2 mu sqrt(3/2) dep_est) (Voigt, 6) and dep / dep_est,
// where dep_est = (q_trial - sigma_y(ep, T)) / (3 mu / J) is the increment without hardening.
// Both scales are exact and cheap; they carry the magnitude, so the targets are O(1) and the
// network only learns the shape of the return. The stress after a return is the difference of
// two numbers up to ~10 sigma_y apart, so a BF16 network that predicted stresses directly would
// carry errors of several per cent of sigma_y. Only plastic states train the network (column 7
// of a target row is its sample weight: 1 plastic, 0 elastic); elastic states never reach it.
//
// Arithmetic. Weights and activations enter the tensor cores as BF16 (mma.sync m16n8k16,
// FP32 accumulation); the optimizer keeps FP32 master weights. One warp owns 16 samples: the
// accumulator fragment of one layer is the A fragment of the next (two 8-column tiles make one
// 16-wide K step), so activations never leave registers in the forward pass. Weight gradients
// are GEMMs over the sample axis: each warp stages its activations and gradients transposed in
// shared memory (BF16) and runs them through the same mma shape; warps sum into FP32 shared
// accumulators and each CTA adds its sums to the global gradient once.
//
// Gate. A particle whose trial von Mises stress is at or below yield takes the exact elastic
// branch (no return exists). Otherwise the prediction is accepted only if (a) dep >= 0,
// (b) the yield function of the predicted stress, |q(tau) - sigma_y(ep + dep)|, and (c) the
// distance of tau from the radial-return stress for the predicted dep,
// |tau - (tau_trial - 2 mu sqrt(3/2) dep n)|, are both within gate_tol * sigma_y0. Every
// rejected particle runs the exact map.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "mpm_b200.h"
#include "mpm_math.h"

namespace surr {

constexpr int kIn = 8, kHid = 64, kOut = 7;
// FP32 parameter vector (out-major weights: W[o][i])
constexpr int kW1 = 0;                   // [64][16] (inputs 8..15 zero)
constexpr int kB1 = kW1 + kHid * 16;     // [64]
constexpr int kW2 = kB1 + kHid;          // [64][64]
constexpr int kB2 = kW2 + kHid * kHid;   // [64]
constexpr int kW3 = kB2 + kHid;          // [8][64] (row 7 zero)
constexpr int kB3 = kW3 + 8 * kHid;      // [8] (entry 7 zero)
constexpr int kParams = kB3 + 8;         // 5768
static_assert(kParams == MPM_SURROGATE_PARAMS, "parameter count");

// BF16 copies for the tensor cores
struct __align__(16) WeightsBf16 {
  __nv_bfloat16 w1f[kHid * 16];   // forward B operand, out-major [o][i]
  __nv_bfloat16 w2f[kHid * kHid];
  __nv_bfloat16 w3f[8 * kHid];
  __nv_bfloat16 w2b[kHid * kHid]; // backward B operand, in-major [i][o]
  __nv_bfloat16 w3b[kHid * 16];   // in-major [i][o], o padded to 16
};

struct Scales {
  float T_lo, T_span, ep;
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ void mma(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A fragment of K columns [16 kc, 16 kc + 16) from two accumulator tiles (2 kc, 2 kc + 1).
__device__ __forceinline__ void chain(const float t[][4], int kc, uint32_t a[4]) {
  a[0] = pack_bf16(t[2 * kc][0], t[2 * kc][1]);
  a[1] = pack_bf16(t[2 * kc][2], t[2 * kc][3]);
  a[2] = pack_bf16(t[2 * kc + 1][0], t[2 * kc + 1][1]);
  a[3] = pack_bf16(t[2 * kc + 1][2], t[2 * kc + 1][3]);
}

// Forward pass of one warp's 16 samples. xa: A fragment of the inputs (K = 16, 8 real).
// h1, h2: post-ReLU activations (accumulator layout, 8 tiles of 8 columns); y: outputs (1 tile).
__device__ __forceinline__ void forward(const WeightsBf16& w, const float* bias, const uint32_t xa[4], float h1[8][4],
                                        float h2[8][4], float y[4], int g, int tig) {
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bias[kB1 + nt * 8 + tig * 2], b1 = bias[kB1 + nt * 8 + tig * 2 + 1];
    h1[nt][0] = b0; h1[nt][1] = b1; h1[nt][2] = b0; h1[nt][3] = b1;
    const __nv_bfloat16* wr = w.w1f + (nt * 8 + g) * 16 + tig * 2;
    mma(h1[nt], xa, ld32(wr), ld32(wr + 8));
#pragma unroll
    for (int j = 0; j < 4; ++j) h1[nt][j] = fmaxf(h1[nt][j], 0.f);
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bias[kB2 + nt * 8 + tig * 2], b1 = bias[kB2 + nt * 8 + tig * 2 + 1];
    h2[nt][0] = b0; h2[nt][1] = b1; h2[nt][2] = b0; h2[nt][3] = b1;
  }
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    uint32_t a[4];
    chain(h1, kc, a);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const __nv_bfloat16* wr = w.w2f + (nt * 8 + g) * kHid + kc * 16 + tig * 2;
      mma(h2[nt], a, ld32(wr), ld32(wr + 8));
    }
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int j = 0; j < 4; ++j) h2[nt][j] = fmaxf(h2[nt][j], 0.f);
  {
    const float b0 = bias[kB3 + tig * 2], b1 = bias[kB3 + tig * 2 + 1];
    y[0] = b0; y[1] = b1; y[2] = b0; y[3] = b1;
  }
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    uint32_t a[4];
    chain(h2, kc, a);
    const __nv_bfloat16* wr = w.w3f + g * kHid + kc * 16 + tig * 2;
    mma(y, a, ld32(wr), ld32(wr + 8));
  }
}

// Per-warp shared staging for the weight-gradient GEMMs: transposed BF16 tiles [feature][sample].
struct WarpStage {
  __nv_bfloat16 xT[16][16];    // inputs (8 real rows)
  __nv_bfloat16 h1T[kHid][16];
  __nv_bfloat16 h2T[kHid][16];
  __nv_bfloat16 d1T[kHid][16]; // dL/d(pre-activation 1)
  __nv_bfloat16 d2T[kHid][16]; // dL/d(pre-activation 2)
  __nv_bfloat16 dyT[16][16];   // dL/dy (7 real rows)
};

constexpr int kTrainThreads = 256;
constexpr int kTrainWarps = kTrainThreads / 32;

struct TrainSmem {
  WeightsBf16 w;
  float bias[kParams];   // only the bias entries are read
  float grad[kParams];   // CTA gradient sums
  WarpStage stage[kTrainWarps];
  float loss[kTrainWarps];
};

// Stores an accumulator tile (16 samples x 8 columns starting at col0) transposed into T[col][s].
__device__ __forceinline__ void store_t(__nv_bfloat16 (*T)[16], const float c[4], int col0, int g, int tig) {
  T[col0 + tig * 2][g] = __float2bfloat16_rn(c[0]);
  T[col0 + tig * 2 + 1][g] = __float2bfloat16_rn(c[1]);
  T[col0 + tig * 2][g + 8] = __float2bfloat16_rn(c[2]);
  T[col0 + tig * 2 + 1][g + 8] = __float2bfloat16_rn(c[3]);
}

// grad[base + o * ld + i] += sum_s A[o][s] B[i][s] for o in [0, M), i in [0, N) (M, N multiples
// of 16 / 8; K = the warp's 16 samples), adding into the CTA's shared accumulators.
template <int M, int N>
__device__ __forceinline__ void wgrad(const __nv_bfloat16 (*A)[16], const __nv_bfloat16 (*B)[16], float* grad, int base,
                                      int ld, int mvalid, int g, int tig) {
#pragma unroll
  for (int mt = 0; mt < M / 16; ++mt) {
    uint32_t a[4];
    a[0] = ld32(&A[mt * 16 + g][tig * 2]);
    a[1] = ld32(&A[mt * 16 + g + 8][tig * 2]);
    a[2] = ld32(&A[mt * 16 + g][tig * 2 + 8]);
    a[3] = ld32(&A[mt * 16 + g + 8][tig * 2 + 8]);
#pragma unroll
    for (int nt = 0; nt < N / 8; ++nt) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
      mma(c, a, ld32(&B[nt * 8 + g][tig * 2]), ld32(&B[nt * 8 + g][tig * 2 + 8]));
      const int o0 = mt * 16 + g, o1 = o0 + 8, i0 = nt * 8 + tig * 2;
      if (o0 < mvalid) {
        atomicAdd(&grad[base + o0 * ld + i0], c[0]);
        atomicAdd(&grad[base + o0 * ld + i0 + 1], c[1]);
      }
      if (o1 < mvalid) {
        atomicAdd(&grad[base + o1 * ld + i0], c[2]);
        atomicAdd(&grad[base + o1 * ld + i0 + 1], c[3]);
      }
    }
  }
}

// Column sums of an accumulator tile over the warp's 16 samples, added to grad[base + col].
__device__ __forceinline__ void bias_grad(const float c[4], float* grad, int base, int col0, int g, int tig,
                                          int valid) {
  float s0 = c[0] + c[2], s1 = c[1] + c[3];
#pragma unroll
  for (int o = 4; o < 32; o <<= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  if (g == 0) {
    if (col0 + tig * 2 < valid) atomicAdd(&grad[base + col0 + tig * 2], s0);
    if (col0 + tig * 2 + 1 < valid) atomicAdd(&grad[base + col0 + tig * 2 + 1], s1);
  }
}

__device__ __forceinline__ void load_weights(WeightsBf16& dst, const WeightsBf16* src) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(&dst);
  for (int i = threadIdx.x; i < (int)(sizeof(WeightsBf16) / 16); i += blockDim.x) d[i] = s[i];
}

// Loss = sum over samples and outputs of wout[o] (y - t)^2 / n_total; gradient into grad_out.
// Samples are rows of X (n x 8) and Y (n x 8, column 7 unused); sample r of this call is row
// (first + r * stride) mod n_data, a strided walk that visits every row once per epoch when
// stride and n_data are coprime.
__global__ void __launch_bounds__(kTrainThreads) k_train(const WeightsBf16* wg, const float* params, const float* X,
                                                         const float* Y, long long n_data, long long first,
                                                         long long stride, int batch, float inv_batch, const float* wout,
                                                         float* grad_out, float* loss_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainSmem& sm = *reinterpret_cast<TrainSmem*>(smem_raw);
  load_weights(sm.w, wg);
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
    sm.bias[i] = params[i];
    sm.grad[i] = 0.f;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  if (lane == 0) sm.loss[warp] = 0.f;
  __syncthreads();
  WarpStage& st = sm.stage[warp];
  const int tiles = batch / 16;
  float wo0 = wout[tig * 2], wo1 = wout[tig * 2 + 1];
  for (int tile = blockIdx.x * kTrainWarps + warp; tile < tiles; tile += gridDim.x * kTrainWarps) {
    const long long r0 = (first + (long long)(tile * 16 + g) * stride) % n_data;
    const long long r1 = (first + (long long)(tile * 16 + g + 8) * stride) % n_data;
    uint32_t xa[4];
    {
      const float2 x0 = *reinterpret_cast<const float2*>(X + r0 * kIn + tig * 2);
      const float2 x1 = *reinterpret_cast<const float2*>(X + r1 * kIn + tig * 2);
      xa[0] = pack_bf16(x0.x, x0.y);
      xa[1] = pack_bf16(x1.x, x1.y);
      xa[2] = 0u;
      xa[3] = 0u;
      st.xT[tig * 2][g] = __float2bfloat16_rn(x0.x);
      st.xT[tig * 2 + 1][g] = __float2bfloat16_rn(x0.y);
      st.xT[tig * 2][g + 8] = __float2bfloat16_rn(x1.x);
      st.xT[tig * 2 + 1][g + 8] = __float2bfloat16_rn(x1.y);
    }
    float h1[8][4], h2[8][4], y[4];
    forward(sm.w, sm.bias, xa, h1, h2, y, g, tig);
    // dL/dy = 2 w (y - t) / batch; output 7 is padding
    float dy[4];
    {
      const float2 t0 = *reinterpret_cast<const float2*>(Y + r0 * 8 + tig * 2);
      const float2 t1 = *reinterpret_cast<const float2*>(Y + r1 * 8 + tig * 2);
      // column 7 of a target row is the sample weight (held by the lane with tig 3)
      const float ws0 = __shfl_sync(0xffffffffu, t0.y, (lane & ~3) | 3);
      const float ws1 = __shfl_sync(0xffffffffu, t1.y, (lane & ~3) | 3);
      const float e0 = y[0] - t0.x, e1 = y[1] - t0.y, e2 = y[2] - t1.x, e3 = y[3] - t1.y;
      const bool pad = tig == 3;  // column 7
      const float w1m = pad ? 0.f : wo1;
      dy[0] = 2.f * wo0 * ws0 * e0 * inv_batch;
      dy[1] = 2.f * w1m * ws0 * e1 * inv_batch;
      dy[2] = 2.f * wo0 * ws1 * e2 * inv_batch;
      dy[3] = 2.f * w1m * ws1 * e3 * inv_batch;
      float l = ws0 * (wo0 * e0 * e0 + w1m * e1 * e1) + ws1 * (wo0 * e2 * e2 + w1m * e3 * e3);
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
      if (lane == 0) sm.loss[warp] += l * inv_batch;
    }
    // dL/dh2 = dy W3 (K = outputs, 8 of 16), masked by ReLU
    float d2[8][4];
    {
      uint32_t a[4] = {pack_bf16(dy[0], dy[1]), pack_bf16(dy[2], dy[3]), 0u, 0u};
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        d2[nt][0] = d2[nt][1] = d2[nt][2] = d2[nt][3] = 0.f;
        mma(d2[nt], a, ld32(sm.w.w3b + (nt * 8 + g) * 16 + tig * 2), 0u);
#pragma unroll
        for (int j = 0; j < 4; ++j) d2[nt][j] = h2[nt][j] > 0.f ? d2[nt][j] : 0.f;
      }
    }
    // dL/dh1 = d2 W2, masked
    float d1[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) d1[nt][0] = d1[nt][1] = d1[nt][2] = d1[nt][3] = 0.f;
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
      uint32_t a[4];
      chain(d2, kc, a);
#pragma unroll
      for (int nt = 0; nt < 8; ++nt) {
        const __nv_bfloat16* wr = sm.w.w2b + (nt * 8 + g) * kHid + kc * 16 + tig * 2;
        mma(d1[nt], a, ld32(wr), ld32(wr + 8));
      }
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int j = 0; j < 4; ++j) d1[nt][j] = h1[nt][j] > 0.f ? d1[nt][j] : 0.f;
    // stage transposed tiles for the weight gradients
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      store_t(st.h1T, h1[nt], nt * 8, g, tig);
      store_t(st.h2T, h2[nt], nt * 8, g, tig);
      store_t(st.d1T, d1[nt], nt * 8, g, tig);
      store_t(st.d2T, d2[nt], nt * 8, g, tig);
    }
    store_t(st.dyT, dy, 0, g, tig);
    for (int i = lane; i < 8 * 16; i += 32) {
      (&st.xT[8][0])[i] = __float2bfloat16_rn(0.f);
      (&st.dyT[8][0])[i] = __float2bfloat16_rn(0.f);
    }
    __syncwarp();
    // dW3[o][i] = sum_s dy[s][o] h2[s][i]; dW2 = d2^T h1; dW1 = d1^T x
    wgrad<16, kHid>(st.dyT, st.h2T, sm.grad, kW3, kHid, kOut, g, tig);
    wgrad<kHid, kHid>(st.d2T, st.h1T, sm.grad, kW2, kHid, kHid, g, tig);
    wgrad<kHid, 8>(st.d1T, st.xT, sm.grad, kW1, 16, kHid, g, tig);
    bias_grad(dy, sm.grad, kB3, 0, g, tig, kOut);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      bias_grad(d2[nt], sm.grad, kB2, nt * 8, g, tig, kHid);
      bias_grad(d1[nt], sm.grad, kB1, nt * 8, g, tig, kHid);
    }
    __syncwarp();
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
    const float v = sm.grad[i];
    if (v != 0.f) atomicAdd(&grad_out[i], v);
  }
  if (threadIdx.x < kTrainWarps && sm.loss[threadIdx.x] != 0.f) atomicAdd(loss_out, sm.loss[threadIdx.x]);
}

// AdamW on the FP32 master parameters, then the BF16 copies (padding entries stay zero).
__global__ void k_adamw(float* params, float* grad, float* m, float* v, int t, float lr, float b1, float b2, float eps,
                        float wd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kParams) return;
  const bool is_w = (i < kB1) || (i >= kW2 && i < kB2) || (i >= kW3 && i < kB3);
  const float gi = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.f - powf(b1, (float)t)), vh = vi / (1.f - powf(b2, (float)t));
  float p = params[i];
  if (is_w) p -= lr * wd * p;
  p -= lr * mh / (sqrtf(vh) + eps);
  params[i] = p;
  grad[i] = 0.f;
}

// Zero the padding of the parameter vector (inputs 8..15 of W1, row 7 of W3, b3[7]).
__global__ void k_pad_zero(float* params) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kHid * 8) params[kW1 + (i >> 3) * 16 + 8 + (i & 7)] = 0.f;
  if (i < kHid) params[kW3 + 7 * kHid + i] = 0.f;
  if (i == 0) params[kB3 + 7] = 0.f;
}

__global__ void k_to_bf16(const float* params, WeightsBf16* w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kHid * kHid; i += gridDim.x * blockDim.x) {
    const int o = i / kHid, in = i % kHid;
    w->w2f[i] = __float2bfloat16_rn(params[kW2 + i]);
    w->w2b[in * kHid + o] = __float2bfloat16_rn(params[kW2 + i]);
    if (i < kHid * 16) {
      w->w1f[i] = __float2bfloat16_rn(params[kW1 + i]);
      const int ii = i / 16, oo = i % 16;  // w3b[i][o]
      w->w3b[i] = __float2bfloat16_rn(oo < 8 ? params[kW3 + oo * kHid + ii] : 0.f);
    }
    if (i < 8 * kHid) w->w3f[i] = __float2bfloat16_rn(params[kW3 + i]);
  }
}

// ---------------------------------------------------------------------------------------------
// Samples and features

__device__ __forceinline__ unsigned mix32(unsigned x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}
__device__ __forceinline__ float urand(unsigned long long seed, long long i, int k) {
  const unsigned h = mix32(mix32(static_cast<unsigned>(seed) ^ mix32(static_cast<unsigned>(i))) ^
                           mix32(static_cast<unsigned>(i >> 32) + 0x9e3779b9u * (k + 1)) ^ static_cast<unsigned>(seed >> 32));
  return (h >> 8) * (1.f / 16777216.f);
}

struct SampleSpec {
  float strain_lo, strain_hi;  // log-uniform magnitude of the principal trial log strains
  float T_lo, T_hi, ep_hi;
  unsigned long long seed;
};

// Trial Hencky strain of F (Voigt, shear components scaled by sqrt 2) from D = F - I.
__device__ void trial_strain(const float D[9], float L6[6]) {
  const mpm::Sym3 B = mpm::cauchy_green_minus_identity(D);
  const int nt = mpm::series_terms(mpm::sym_norm(B));
  mpm::Sym3 L;
  if (nt > 0) {
    L = mpm::matrix_series<0>(B, nt);
    L.xx *= .5f; L.yy *= .5f; L.zz *= .5f; L.xy *= .5f; L.xz *= .5f; L.yz *= .5f;
  } else {
    float beta[3], U[9], e[3];
    mpm::sym_eig3(B, beta, U);
    for (int k = 0; k < 3; ++k) e[k] = mpm::hencky_strain(beta[k]);
    L = mpm::rotate_diag(U, e);
  }
  const float r2 = 1.41421356237f;
  L6[0] = L.xx; L6[1] = L.yy; L6[2] = L.zz; L6[3] = r2 * L.xy; L6[4] = r2 * L.xz; L6[5] = r2 * L.yz;
}

// One random trial state: F = R diag(exp e) R^T with |e| log-uniform and a random direction,
// ep and T uniform.
__device__ void random_state(const SampleSpec& sp, long long i, float D[9], float& ep, float& T) {
  const float u0 = urand(sp.seed, i, 0);
  const float mag = expf(logf(sp.strain_lo) + u0 * (logf(sp.strain_hi) - logf(sp.strain_lo)));
  // direction of the principal strains: uniform on the sphere
  const float z = 2.f * urand(sp.seed, i, 1) - 1.f, ph = 6.283185307f * urand(sp.seed, i, 2);
  const float rxy = sqrtf(fmaxf(0.f, 1.f - z * z));
  const float e[3] = {mag * rxy * cosf(ph), mag * rxy * sinf(ph), mag * z};
  // random rotation from a uniform unit quaternion
  const float a1 = urand(sp.seed, i, 3), a2 = 6.283185307f * urand(sp.seed, i, 4), a3 = 6.283185307f * urand(sp.seed, i, 5);
  const float s1 = sqrtf(1.f - a1), s2 = sqrtf(a1);
  const float qw = s1 * sinf(a2), qx = s1 * cosf(a2), qy = s2 * sinf(a3), qz = s2 * cosf(a3);
  const float R[9] = {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw),
                      2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw),
                      2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)};
  const float s[3] = {expm1f(e[0]), expm1f(e[1]), expm1f(e[2])};
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) D[a * 3 + b] = R[a * 3 + 0] * s[0] * R[b * 3 + 0] + R[a * 3 + 1] * s[1] * R[b * 3 + 1] +
                                               R[a * 3 + 2] * s[2] * R[b * 3 + 2];
  ep = sp.ep_hi * urand(sp.seed, i, 6);
  T = sp.T_lo + (sp.T_hi - sp.T_lo) * urand(sp.seed, i, 7);
}

// Trial invariants of the J2 return (src/three/metal-plasticity.js:20-27 in SI form).
struct Trial {
  float dv[6];   // dev L in Voigt order (shear scaled by sqrt 2)
  float len;     // |dev L|
  float trL, J, q, soft, yield, hard, dep_est;
};

__device__ Trial trial_of(const mpm::MaterialDev& mt, const float L6[6], float T, float ep) {
  Trial t;
  t.trL = L6[0] + L6[1] + L6[2];
  const float tr3 = t.trL * (1.f / 3.f);
  t.dv[0] = L6[0] - tr3; t.dv[1] = L6[1] - tr3; t.dv[2] = L6[2] - tr3;
  t.dv[3] = L6[3]; t.dv[4] = L6[4]; t.dv[5] = L6[5];
  t.len = sqrtf(t.dv[0] * t.dv[0] + t.dv[1] * t.dv[1] + t.dv[2] * t.dv[2] + t.dv[3] * t.dv[3] + t.dv[4] * t.dv[4] +
                t.dv[5] * t.dv[5]);
  t.J = fmaxf(1e-6f, expf(t.trL));
  t.q = 2.449489742783178f * mt.mu * t.len / t.J;
  t.soft = 1.f;
  if (mt.model == 10) t.soft = 1.f - (1.f - mt.hot_ratio) * fminf(1.f, fmaxf(0.f, (T - mt.T_ref) * mt.inv_T_span));
  t.hard = mt.model == 4 ? 0.f : mt.hardening;
  t.yield = (mt.yield_stress + t.hard * ep) * t.soft;
  t.dep_est = (t.q - t.yield) * t.J / (3.f * mt.mu);
  return t;
}

__device__ void features(const Scales& sc, const Trial& t, float T, float ep, float x[8]) {
  const float il = t.len > 0.f ? 1.f / t.len : 0.f;
  for (int k = 0; k < 6; ++k) x[k] = t.dv[k] * il;
  x[6] = (T - sc.T_lo) / sc.T_span;
  x[7] = ep / sc.ep;
}

__device__ void trial_stress(const mpm::MaterialDev& mt, const float L6[6], float t6[6]) {
  const float tr = L6[0] + L6[1] + L6[2];
  for (int k = 0; k < 6; ++k) t6[k] = 2.f * mt.mu * L6[k];
  for (int k = 0; k < 3; ++k) t6[k] += mt.lam * tr;
}

// Training rows: X (8 features) and Y (7 targets + pad) from the exact map on random states.
__global__ void k_samples(mpm::MaterialDev mt, Scales sc, SampleSpec sp, long long n, float* X, float* Y, float* Dout,
                          float* epout, float* Tout) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float D[9], ep, T;
    random_state(sp, i, D, ep, T);
    if (Dout) {
      for (int k = 0; k < 9; ++k) Dout[i * 9 + k] = D[k];
      epout[i] = ep;
      Tout[i] = T;
    }
    float L6[6], x[8], t6[6];
    trial_strain(D, L6);
    const Trial tr = trial_of(mt, L6, T, ep);
    features(sc, tr, T, ep, x);
    trial_stress(mt, L6, t6);
    const mpm::ConstitutiveOut co = mpm::constitutive_update(mt, D, ep, T, 0.f, true);
    const float r2 = 1.41421356237f;
    const float tau6[6] = {co.tau.xx, co.tau.yy, co.tau.zz, r2 * co.tau.xy, r2 * co.tau.xz, r2 * co.tau.yz};
    const bool plastic = tr.q > tr.yield && tr.dep_est > 0.f;
    const float sd = plastic ? 1.f / (2.f * mt.mu * 1.224744871391589f * tr.dep_est) : 0.f;
    for (int k = 0; k < 8; ++k) X[i * 8 + k] = x[k];
    for (int k = 0; k < 6; ++k) Y[i * 8 + k] = (tau6[k] - t6[k]) * sd;
    Y[i * 8 + 6] = plastic ? co.dep / tr.dep_est : 0.f;
    Y[i * 8 + 7] = plastic ? 1.f : 0.f;  // sample weight
  }
}

// Plain forward of rows of X into Y (7 outputs + pad): one warp per 16 rows.
__global__ void __launch_bounds__(256) k_forward(const WeightsBf16* wg, const float* params, const float* X, long long n,
                                                 float* Yout) {
  __shared__ WeightsBf16 w;
  __shared__ float bias[kParams];
  load_weights(w, wg);
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) bias[i] = params[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  const long long tiles = (n + 15) / 16;
  for (long long tile = blockIdx.x * 8ll + warp; tile < tiles; tile += gridDim.x * 8ll) {
    const long long r0 = tile * 16 + g, r1 = r0 + 8;
    float2 x0 = make_float2(0.f, 0.f), x1 = x0;
    if (r0 < n) x0 = *reinterpret_cast<const float2*>(X + r0 * kIn + tig * 2);
    if (r1 < n) x1 = *reinterpret_cast<const float2*>(X + r1 * kIn + tig * 2);
    const uint32_t xa[4] = {pack_bf16(x0.x, x0.y), pack_bf16(x1.x, x1.y), 0u, 0u};
    float h1[8][4], h2[8][4], y[4];
    forward(w, bias, xa, h1, h2, y, g, tig);
    if (r0 < n) *reinterpret_cast<float2*>(Yout + r0 * 8 + tig * 2) = make_float2(y[0], y[1]);
    if (r1 < n) *reinterpret_cast<float2*>(Yout + r1 * 8 + tig * 2) = make_float2(y[2], y[3]);
  }
}

// ---------------------------------------------------------------------------------------------
// Gated return map over particles. Each thread owns one particle; the warp's 32 particles go
// through the MLP as two 16-row tiles staged in shared memory.

constexpr int kGateThreads = 256;

struct GateSmem {
  WeightsBf16 w;
  float bias[kParams];
  float x[kGateThreads][8];
  float y[kGateThreads][8];
};

struct GateOut {
  unsigned elastic, learned, fallback;
};

// D = F - I (n x 9 float, formed by the caller in higher precision), ep, T in; D, dep and tau
// (n x 6: xx yy zz xy xz yz) out; path: 0 elastic, 1 learned, 2 exact fallback. use_mlp = 0 runs
// the exact map for every particle through the same kernel, so both timings share loads and stores.
__global__ void __launch_bounds__(kGateThreads) k_gated(const WeightsBf16* wg, const float* params, mpm::MaterialDev mt,
                                                        Scales sc, float gate_tol, int use_mlp, long long n,
                                                        const float* Din, const float* epin, const float* Tin, float* Dout,
                                                        float* dep, float* tau, signed char* path, GateOut* counts) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GateSmem& sm = *reinterpret_cast<GateSmem*>(smem_raw);
  if (use_mlp) {
    load_weights(sm.w, wg);
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) sm.bias[i] = params[i];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  unsigned c_el = 0, c_ml = 0, c_fb = 0;
  const float r2 = 1.41421356237f, ir2 = 0.70710678118f, s15 = 1.224744871391589f;
  for (long long base = (long long)blockIdx.x * kGateThreads; base < n; base += (long long)gridDim.x * kGateThreads) {
    const long long i = base + threadIdx.x;
    const bool live = i < n;
    float D[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, ep = 0.f, T = 0.f, L6[6] = {0, 0, 0, 0, 0, 0};
    if (live) {
      for (int k = 0; k < 9; ++k) D[k] = Din[i * 9 + k];
      ep = epin ? epin[i] : 0.f;
      T = Tin ? Tin[i] : 0.f;
      trial_strain(D, L6);
    }
    const Trial tr = trial_of(mt, L6, T, ep);
    // the gate's first decision is the exact one: below yield there is no return
    const bool plastic = live && tr.q > tr.yield;
    bool accepted = false;
    float tau6[6], dp = 0.f;
    if (use_mlp && __any_sync(0xffffffffu, plastic)) {
      float x[8];
      features(sc, tr, T, ep, x);
      for (int k = 0; k < 8; ++k) sm.x[threadIdx.x][k] = x[k];
      __syncwarp();
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const int row0 = warp * 32 + half * 16;
        const float2 x0 = *reinterpret_cast<const float2*>(&sm.x[row0 + g][tig * 2]);
        const float2 x1 = *reinterpret_cast<const float2*>(&sm.x[row0 + g + 8][tig * 2]);
        const uint32_t xa[4] = {pack_bf16(x0.x, x0.y), pack_bf16(x1.x, x1.y), 0u, 0u};
        float h1[8][4], h2[8][4], y[4];
        forward(sm.w, sm.bias, xa, h1, h2, y, g, tig);
        *reinterpret_cast<float2*>(&sm.y[row0 + g][tig * 2]) = make_float2(y[0], y[1]);
        *reinterpret_cast<float2*>(&sm.y[row0 + g + 8][tig * 2]) = make_float2(y[2], y[3]);
      }
      __syncwarp();
      if (plastic) {
        float t6[6];
        trial_stress(mt, L6, t6);
        const float smag = 2.f * mt.mu * s15 * tr.dep_est;
        for (int k = 0; k < 6; ++k) tau6[k] = t6[k] + smag * sm.y[threadIdx.x][k];
        dp = tr.dep_est * sm.y[threadIdx.x][6];
        // residuals of the prediction against the return's two defining equations
        const float y0 = fmaxf(mt.yield_stress * tr.soft, 1e-30f);
        const float p3 = (tau6[0] + tau6[1] + tau6[2]) * (1.f / 3.f);
        const float s0 = tau6[0] - p3, s1 = tau6[1] - p3, s2 = tau6[2] - p3;
        const float sq = s0 * s0 + s1 * s1 + s2 * s2 + tau6[3] * tau6[3] + tau6[4] * tau6[4] + tau6[5] * tau6[5];
        const float q_pred = s15 * sqrtf(sq) / tr.J;
        const float r_yield = fabsf(q_pred - (mt.yield_stress + tr.hard * (ep + dp)) * tr.soft) / y0;
        const float k2 = 2.f * mt.mu * s15 * dp / fmaxf(tr.len, 1e-20f);
        float r_flow = 0.f;
        for (int k = 0; k < 6; ++k) {
          const float d = tau6[k] - (t6[k] - k2 * tr.dv[k]);
          r_flow += d * d;
        }
        r_flow = sqrtf(r_flow) / y0;
        accepted = dp >= 0.f && r_yield <= gate_tol && r_flow <= gate_tol;
      }
    }
    if (live) {
      if (!plastic) {
        const mpm::ConstitutiveOut co = mpm::constitutive_update(mt, D, ep, T, 0.f, false);
        tau6[0] = co.tau.xx; tau6[1] = co.tau.yy; tau6[2] = co.tau.zz;
        tau6[3] = co.tau.xy * r2; tau6[4] = co.tau.xz * r2; tau6[5] = co.tau.yz * r2;
        dp = 0.f;
        ++c_el;
        if (path) path[i] = 0;
      } else if (accepted) {
        // the predicted increment returns F: F' = exp((scale - 1) dev L) F
        const float scale = fmaxf(0.f, 1.f - s15 * dp / fmaxf(tr.len, 1e-20f));
        const float gs = scale - 1.f;
        const mpm::Sym3 M{gs * tr.dv[0], gs * tr.dv[1], gs * tr.dv[2], gs * tr.dv[3] * ir2, gs * tr.dv[4] * ir2,
                          gs * tr.dv[5] * ir2};
        const int nm = mpm::series_terms(mpm::sym_norm(M));
        const mpm::Sym3 E = mpm::matrix_series<2>(M, nm > 0 ? nm : 10);
        float Dn[9];
        for (int b = 0; b < 3; ++b) {
          Dn[0 * 3 + b] = E.xx * D[0 * 3 + b] + E.xy * D[1 * 3 + b] + E.xz * D[2 * 3 + b];
          Dn[1 * 3 + b] = E.xy * D[0 * 3 + b] + E.yy * D[1 * 3 + b] + E.yz * D[2 * 3 + b];
          Dn[2 * 3 + b] = E.xz * D[0 * 3 + b] + E.yz * D[1 * 3 + b] + E.zz * D[2 * 3 + b];
        }
        D[0] += Dn[0] + E.xx; D[1] += Dn[1] + E.xy; D[2] += Dn[2] + E.xz;
        D[3] += Dn[3] + E.xy; D[4] += Dn[4] + E.yy; D[5] += Dn[5] + E.yz;
        D[6] += Dn[6] + E.xz; D[7] += Dn[7] + E.yz; D[8] += Dn[8] + E.zz;
        ++c_ml;
        if (path) path[i] = 1;
      } else {
        const mpm::ConstitutiveOut co = mpm::constitutive_update(mt, D, ep, T, 0.f, true);
        tau6[0] = co.tau.xx; tau6[1] = co.tau.yy; tau6[2] = co.tau.zz;
        tau6[3] = co.tau.xy * r2; tau6[4] = co.tau.xz * r2; tau6[5] = co.tau.yz * r2;
        dp = co.dep;
        ++c_fb;
        if (path) path[i] = 2;
      }
      for (int k = 0; k < 9; ++k) Dout[i * 9 + k] = D[k];
      dep[i] = dp;
      tau[i * 6 + 0] = tau6[0]; tau[i * 6 + 1] = tau6[1]; tau[i * 6 + 2] = tau6[2];
      tau[i * 6 + 3] = tau6[3] * ir2; tau[i * 6 + 4] = tau6[4] * ir2; tau[i * 6 + 5] = tau6[5] * ir2;
    }
    __syncwarp();
  }
  if (counts) {
    for (int o = 16; o; o >>= 1) {
      c_el += __shfl_xor_sync(0xffffffffu, c_el, o);
      c_ml += __shfl_xor_sync(0xffffffffu, c_ml, o);
      c_fb += __shfl_xor_sync(0xffffffffu, c_fb, o);
    }
    if (lane == 0) {
      atomicAdd(&counts->elastic, c_el);
      atomicAdd(&counts->learned, c_ml);
      atomicAdd(&counts->fallback, c_fb);
    }
  }
}

mpm::MaterialDev to_dev(const mpm_material& m) {
  mpm::MaterialDev d{};
  d.model = m.model;
  d.mu = (float)m.mu;
  d.lam = (float)m.lambda;
  d.yield_stress = (float)m.yield_stress;
  d.hardening = (float)m.hardening;
  d.T_ref = (float)m.T_ref;
  d.inv_T_span = m.T_hot > m.T_ref ? (float)(1.0 / (m.T_hot - m.T_ref)) : 0.f;
  d.hot_ratio = (float)m.hot_ratio;
  d.heat_per_work = m.specific_heat > 0 ? (float)(m.heat_fraction / m.specific_heat) : 0.f;
  d.wave_modulus = (float)(m.lambda + 2 * m.mu);
  return d;
}

}  // namespace surr

struct mpm_surrogate {
  mpm_material mat{};
  mpm::MaterialDev mt{};
  surr::Scales sc{};
  surr::SampleSpec spec{};
  cudaStream_t stream = nullptr;
  float* params = nullptr;  // FP32 master
  float* grad = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  float* loss = nullptr;
  surr::WeightsBf16* wbf = nullptr;
  int num_sms = 148;
  int adam_t = 0;
  std::string err;
};

namespace {

int sfail(mpm_surrogate* s, int rc, const std::string& why) {
  if (s) s->err = why;
  return rc;
}

#define SCUDA(s, call)                                                                             \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess) return sfail(s, e_ == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA, \
                                        std::string(#call) + ": " + cudaGetErrorString(e_));       \
  } while (0)

int sync_bf16(mpm_surrogate* s) {
  surr::k_pad_zero<<<2, 256, 0, s->stream>>>(s->params);
  surr::k_to_bf16<<<16, 256, 0, s->stream>>>(s->params, s->wbf);
  SCUDA(s, cudaGetLastError());
  return MPM_OK;
}

}  // namespace

extern "C" {

int mpm_surrogate_create(const mpm_material* material, uint64_t seed, mpm_surrogate** out) {
  if (!material || !out) return MPM_ERR_INVALID_ARG;
  *out = nullptr;
  if (material->model != 4 && material->model != 5 && material->model != 10) return MPM_ERR_UNSUPPORTED;
  if (!(material->mu > 0) || !(material->yield_stress > 0)) return MPM_ERR_INVALID_ARG;
  mpm_surrogate* s = new mpm_surrogate();
  s->mat = *material;
  s->mt = surr::to_dev(*material);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, dev);
  auto bail = [&](int rc) {
    mpm_surrogate_destroy(s);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(MPM_ERR_CUDA);
  const size_t pb = surr::kParams * sizeof(float);
  if (cudaMalloc(&s->params, pb) != cudaSuccess || cudaMalloc(&s->grad, pb) != cudaSuccess ||
      cudaMalloc(&s->adam_m, pb) != cudaSuccess || cudaMalloc(&s->adam_v, pb) != cudaSuccess ||
      cudaMalloc(&s->loss, 16) != cudaSuccess || cudaMalloc(&s->wbf, sizeof(surr::WeightsBf16)) != cudaSuccess)
    return bail(MPM_ERR_OUT_OF_MEMORY);
  if (cudaFuncSetAttribute(surr::k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(surr::TrainSmem)) !=
          cudaSuccess ||
      cudaFuncSetAttribute(surr::k_gated, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(surr::GateSmem)) !=
          cudaSuccess)
    return bail(MPM_ERR_CUDA);
  // He initialisation from a seeded host generator (fan-in 8, 64, 64), zero biases
  std::vector<float> p(surr::kParams, 0.f);
  uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto nrm = [&]() {
    double u[2];
    for (double& x : u) {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      x = ((st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }
    return std::sqrt(-2.0 * std::log(u[0])) * std::cos(6.283185307179586 * u[1]);
  };
  for (int o = 0; o < surr::kHid; ++o)
    for (int i = 0; i < surr::kIn; ++i) p[surr::kW1 + o * 16 + i] = (float)(nrm() * std::sqrt(2.0 / surr::kIn));
  for (int k = 0; k < surr::kHid * surr::kHid; ++k) p[surr::kW2 + k] = (float)(nrm() * std::sqrt(2.0 / surr::kHid));
  for (int o = 0; o < surr::kOut; ++o)
    for (int i = 0; i < surr::kHid; ++i) p[surr::kW3 + o * surr::kHid + i] = (float)(nrm() * std::sqrt(1.0 / surr::kHid));
  if (cudaMemcpy(s->params, p.data(), pb, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(s->grad, 0, pb) != cudaSuccess || cudaMemset(s->adam_m, 0, pb) != cudaSuccess ||
      cudaMemset(s->adam_v, 0, pb) != cudaSuccess)
    return bail(MPM_ERR_CUDA);
  // feature and target scales
  s->sc.T_lo = 293.f;
  s->sc.T_span = 307.f;
  s->sc.ep = 0.2f;
  if (sync_bf16(s) != MPM_OK || cudaStreamSynchronize(s->stream) != cudaSuccess) return bail(MPM_ERR_CUDA);
  *out = s;
  return MPM_OK;
}

int mpm_surrogate_destroy(mpm_surrogate* s) {
  if (!s) return MPM_ERR_INVALID_ARG;
  if (s->stream) cudaStreamSynchronize(s->stream);
  void* bufs[] = {s->params, s->grad, s->adam_m, s->adam_v, s->loss, s->wbf};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return MPM_OK;
}

const char* mpm_surrogate_last_error(const mpm_surrogate* s) { return s ? s->err.c_str() : "null handle"; }

int mpm_surrogate_get_weights(mpm_surrogate* s, float* params) {
  if (!s || !params) return MPM_ERR_INVALID_ARG;
  SCUDA(s, cudaMemcpyAsync(params, s->params, surr::kParams * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  SCUDA(s, cudaStreamSynchronize(s->stream));
  return MPM_OK;
}

int mpm_surrogate_set_weights(mpm_surrogate* s, const float* params) {
  if (!s || !params) return MPM_ERR_INVALID_ARG;
  SCUDA(s, cudaMemcpyAsync(s->params, params, surr::kParams * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  int rc = sync_bf16(s);
  if (rc) return rc;
  SCUDA(s, cudaStreamSynchronize(s->stream));
  return MPM_OK;
}

int mpm_surrogate_samples(mpm_surrogate* s, const mpm_surrogate_config* cfg, int64_t n, float* X, float* Y, double* F,
                          double* ep, double* T) {
  if (!s || !cfg || n <= 0 || !X || !Y) return MPM_ERR_INVALID_ARG;
  surr::SampleSpec sp{(float)cfg->strain_min, (float)cfg->strain_max, (float)cfg->T_min, (float)cfg->T_max,
                      (float)cfg->ep_max, cfg->seed};
  float *dX = nullptr, *dY = nullptr, *dD = nullptr, *dep = nullptr, *dT = nullptr;
  SCUDA(s, cudaMalloc(&dX, n * 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&dY, n * 8 * sizeof(float)));
  if (F) {
    SCUDA(s, cudaMalloc(&dD, n * 9 * sizeof(float)));
    SCUDA(s, cudaMalloc(&dep, n * sizeof(float)));
    SCUDA(s, cudaMalloc(&dT, n * sizeof(float)));
  }
  surr::k_samples<<<s->num_sms * 8, 256, 0, s->stream>>>(s->mt, s->sc, sp, n, dX, dY, dD, dep, dT);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(X, dX, n * 8 * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Y, dY, n * 8 * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  std::vector<float> hD, hep, hT;
  if (F && e == cudaSuccess) {
    hD.resize(n * 9);
    hep.resize(n);
    hT.resize(n);
    e = cudaMemcpyAsync(hD.data(), dD, n * 9 * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hep.data(), dep, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hT.data(), dT, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(dX);
  cudaFree(dY);
  if (dD) cudaFree(dD);
  if (dep) cudaFree(dep);
  if (dT) cudaFree(dT);
  if (e != cudaSuccess) return sfail(s, MPM_ERR_CUDA, cudaGetErrorString(e));
  if (F) {
    for (int64_t i = 0; i < n * 9; ++i) F[i] = (double)hD[i] + ((i % 9) % 4 == 0 ? 1.0 : 0.0);
    if (ep)
      for (int64_t i = 0; i < n; ++i) ep[i] = hep[i];
    if (T)
      for (int64_t i = 0; i < n; ++i) T[i] = hT[i];
  }
  return MPM_OK;
}

int mpm_surrogate_train(mpm_surrogate* s, const mpm_surrogate_config* cfg, float* loss_history) {
  if (!s || !cfg) return MPM_ERR_INVALID_ARG;
  if (cfg->samples < 16 || cfg->batch < 16 || cfg->batch % 16 || cfg->steps <= 0 || !(cfg->lr > 0))
    return sfail(s, MPM_ERR_INVALID_ARG, "samples >= 16, batch a multiple of 16, steps > 0, lr > 0");
  const long long n = cfg->samples;
  float *X = nullptr, *Y = nullptr, *wout = nullptr;
  SCUDA(s, cudaMalloc(&X, n * 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&Y, n * 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&wout, 8 * sizeof(float)));
  const float w[8] = {1, 1, 1, 1, 1, 1, (float)(cfg->dep_weight > 0 ? cfg->dep_weight : 1.0), 0};
  surr::SampleSpec sp{(float)cfg->strain_min, (float)cfg->strain_max, (float)cfg->T_min, (float)cfg->T_max,
                      (float)cfg->ep_max, cfg->seed};
  int rc = MPM_OK;
  cudaError_t e = cudaMemcpyAsync(wout, w, sizeof w, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) {
    surr::k_samples<<<s->num_sms * 8, 256, 0, s->stream>>>(s->mt, s->sc, sp, n, X, Y, nullptr, nullptr, nullptr);
    e = cudaGetLastError();
  }
  // stride coprime with n walks every sample once per epoch in a scattered order
  long long stride = 2654435761ll % n;
  auto gcd = [](long long a, long long b) {
    while (b) {
      const long long t = a % b;
      a = b;
      b = t;
    }
    return a;
  };
  if (stride < 1) stride = 1;
  while (gcd(stride, n) != 1) ++stride;
  std::vector<float> hist(cfg->steps, 0.f);
  float* dloss = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&dloss, cfg->steps * sizeof(float));
  if (e == cudaSuccess) e = cudaMemsetAsync(dloss, 0, cfg->steps * sizeof(float), s->stream);
  long long first = 0;
  for (int t = 0; t < cfg->steps && e == cudaSuccess && rc == MPM_OK; ++t) {
    const float lr_scale = cfg->cosine ? 0.5f * (1.f + cosf(3.14159265f * t / cfg->steps)) : 1.f;
    mpm_surrogate_config c = *cfg;
    c.lr = cfg->lr * lr_scale;
    const int tiles = cfg->batch / 16;
    const int blocks = std::min(s->num_sms, (tiles + surr::kTrainWarps - 1) / surr::kTrainWarps);
    surr::k_train<<<blocks, surr::kTrainThreads, sizeof(surr::TrainSmem), s->stream>>>(
        s->wbf, s->params, X, Y, n, first, stride, cfg->batch, 1.f / cfg->batch, wout, s->grad, dloss + t);
    ++s->adam_t;
    surr::k_adamw<<<(surr::kParams + 255) / 256, 256, 0, s->stream>>>(s->params, s->grad, s->adam_m, s->adam_v,
                                                                       s->adam_t, (float)c.lr, 0.9f, 0.999f, 1e-8f,
                                                                       (float)cfg->weight_decay);
    rc = sync_bf16(s);
    first = (first + (long long)cfg->batch * stride) % n;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && rc == MPM_OK)
    e = cudaMemcpyAsync(hist.data(), dloss, cfg->steps * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(X);
  cudaFree(Y);
  cudaFree(wout);
  if (dloss) cudaFree(dloss);
  if (rc != MPM_OK) return rc;
  if (e != cudaSuccess) return sfail(s, MPM_ERR_CUDA, cudaGetErrorString(e));
  if (loss_history) std::memcpy(loss_history, hist.data(), cfg->steps * sizeof(float));
  return MPM_OK;
}

int mpm_surrogate_grad(mpm_surrogate* s, int64_t n, const float* X, const float* Y, const float* out_weight,
                       float* grad, double* loss) {
  if (!s || n < 16 || n % 16 || !X || !Y || !grad) return MPM_ERR_INVALID_ARG;
  float *dX = nullptr, *dY = nullptr, *dw = nullptr, *dl = nullptr;
  SCUDA(s, cudaMalloc(&dX, n * 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&dY, n * 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&dw, 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&dl, sizeof(float)));
  const float w1[8] = {1, 1, 1, 1, 1, 1, 1, 0};
  cudaError_t e = cudaMemcpyAsync(dX, X, n * 8 * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dY, Y, n * 8 * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dw, out_weight ? out_weight : w1, 8 * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(dl, 0, sizeof(float), s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->grad, 0, surr::kParams * sizeof(float), s->stream);
  if (e == cudaSuccess) {
    const int tiles = (int)(n / 16);
    const int blocks = std::min(s->num_sms, (tiles + surr::kTrainWarps - 1) / surr::kTrainWarps);
    surr::k_train<<<blocks, surr::kTrainThreads, sizeof(surr::TrainSmem), s->stream>>>(
        s->wbf, s->params, dX, dY, n, 0, 1, (int)n, 1.f / n, dw, s->grad, dl);
    e = cudaGetLastError();
  }
  float lh = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(grad, s->grad, surr::kParams * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&lh, dl, sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->grad, 0, surr::kParams * sizeof(float), s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(dX);
  cudaFree(dY);
  cudaFree(dw);
  cudaFree(dl);
  if (e != cudaSuccess) return sfail(s, MPM_ERR_CUDA, cudaGetErrorString(e));
  if (loss) *loss = lh;
  return MPM_OK;
}

int mpm_surrogate_forward(mpm_surrogate* s, int64_t n, const float* X, float* Y) {
  if (!s || n <= 0 || !X || !Y) return MPM_ERR_INVALID_ARG;
  float *dX = nullptr, *dY = nullptr;
  SCUDA(s, cudaMalloc(&dX, n * 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&dY, n * 8 * sizeof(float)));
  cudaError_t e = cudaMemcpyAsync(dX, X, n * 8 * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(dY, 0, n * 8 * sizeof(float), s->stream);
  if (e == cudaSuccess) {
    const long long tiles = (n + 15) / 16;
    const int blocks = (int)std::min<long long>(s->num_sms * 4, (tiles + 7) / 8);
    surr::k_forward<<<blocks, 256, 0, s->stream>>>(s->wbf, s->params, dX, n, dY);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(Y, dY, n * 8 * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(dX);
  cudaFree(dY);
  if (e != cudaSuccess) return sfail(s, MPM_ERR_CUDA, cudaGetErrorString(e));
  return MPM_OK;
}

int mpm_return_map_learned(mpm_surrogate* s, int64_t n, const double* F_in, const double* ep, const double* T,
                           double gate_tol, int32_t use_mlp, double* F_out, double* dep, double* tau, int8_t* path,
                           mpm_gate_counts* counts) {
  if (!s || n < 0 || (n > 0 && (!F_in || !F_out || !dep || !tau))) return MPM_ERR_INVALID_ARG;
  if (n == 0) return MPM_OK;
  // D = F - I in double before rounding: at small strains F - I in FP32 would lose digits
  std::vector<float> hF(n * 9), he(n, 0.f), hT(n, 0.f);
  for (int64_t i = 0; i < n * 9; ++i) hF[i] = (float)(F_in[i] - ((i % 9) % 4 == 0 ? 1.0 : 0.0));
  if (ep)
    for (int64_t i = 0; i < n; ++i) he[i] = (float)ep[i];
  if (T)
    for (int64_t i = 0; i < n; ++i) hT[i] = (float)T[i];
  float *dF = nullptr, *de = nullptr, *dT = nullptr, *dFo = nullptr, *ddep = nullptr, *dtau = nullptr;
  signed char* dpath = nullptr;
  surr::GateOut* dc = nullptr;
  SCUDA(s, cudaMalloc(&dF, n * 9 * sizeof(float)));
  SCUDA(s, cudaMalloc(&de, n * sizeof(float)));
  SCUDA(s, cudaMalloc(&dT, n * sizeof(float)));
  SCUDA(s, cudaMalloc(&dFo, n * 9 * sizeof(float)));
  SCUDA(s, cudaMalloc(&ddep, n * sizeof(float)));
  SCUDA(s, cudaMalloc(&dtau, n * 6 * sizeof(float)));
  SCUDA(s, cudaMalloc(&dpath, n));
  SCUDA(s, cudaMalloc(&dc, sizeof(surr::GateOut)));
  cudaError_t e = cudaMemcpyAsync(dF, hF.data(), n * 9 * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(de, he.data(), n * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dT, hT.data(), n * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(dc, 0, sizeof(surr::GateOut), s->stream);
  if (e == cudaSuccess) {
    const int blocks = (int)std::min<long long>(s->num_sms * 4, (n + surr::kGateThreads - 1) / surr::kGateThreads);
    surr::k_gated<<<blocks, surr::kGateThreads, sizeof(surr::GateSmem), s->stream>>>(
        s->wbf, s->params, s->mt, s->sc, (float)gate_tol, use_mlp, n, dF, de, dT, dFo, ddep, dtau, dpath, dc);
    e = cudaGetLastError();
  }
  std::vector<float> oF(n * 9), od(n), ot(n * 6);
  surr::GateOut hc{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(oF.data(), dFo, n * 9 * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(od.data(), ddep, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ot.data(), dtau, n * 6 * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess && path) e = cudaMemcpyAsync(path, dpath, n, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hc, dc, sizeof hc, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  void* bufs[] = {dF, de, dT, dFo, ddep, dtau, dpath, dc};
  for (void* b : bufs) cudaFree(b);
  if (e != cudaSuccess) return sfail(s, MPM_ERR_CUDA, cudaGetErrorString(e));
  for (int64_t i = 0; i < n * 9; ++i) F_out[i] = (double)oF[i] + ((i % 9) % 4 == 0 ? 1.0 : 0.0);
  for (int64_t i = 0; i < n; ++i) dep[i] = od[i];
  for (int64_t i = 0; i < n; ++i) {
    // full 3x3 Kirchhoff stress, row-major
    const float* t = &ot[i * 6];
    const double full[9] = {t[0], t[3], t[4], t[3], t[1], t[5], t[4], t[5], t[2]};
    for (int k = 0; k < 9; ++k) tau[i * 9 + k] = full[k];
  }
  if (counts) {
    counts->elastic = hc.elastic;
    counts->learned = hc.learned;
    counts->fallback = hc.fallback;
  }
  return MPM_OK;
}

// Timing of the gated map against the exact map on n device-resident random trial states.
int mpm_surrogate_time(mpm_surrogate* s, const mpm_surrogate_config* cfg, int64_t n, int32_t iters, double gate_tol,
                       double* ms_exact, double* ms_learned, mpm_gate_counts* counts) {
  if (!s || !cfg || n <= 0 || iters <= 0 || !ms_exact || !ms_learned) return MPM_ERR_INVALID_ARG;
  surr::SampleSpec sp{(float)cfg->strain_min, (float)cfg->strain_max, (float)cfg->T_min, (float)cfg->T_max,
                      (float)cfg->ep_max, cfg->seed};
  float *X = nullptr, *Y = nullptr, *dD = nullptr, *de = nullptr, *dT = nullptr, *dFo = nullptr, *ddep = nullptr,
        *dtau = nullptr;
  surr::GateOut* dc = nullptr;
  SCUDA(s, cudaMalloc(&X, n * 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&Y, n * 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&dD, n * 9 * sizeof(float)));
  SCUDA(s, cudaMalloc(&de, n * sizeof(float)));
  SCUDA(s, cudaMalloc(&dT, n * sizeof(float)));
  SCUDA(s, cudaMalloc(&dFo, n * 9 * sizeof(float)));
  SCUDA(s, cudaMalloc(&ddep, n * sizeof(float)));
  SCUDA(s, cudaMalloc(&dtau, n * 6 * sizeof(float)));
  SCUDA(s, cudaMalloc(&dc, sizeof(surr::GateOut)));
  surr::k_samples<<<s->num_sms * 8, 256, 0, s->stream>>>(s->mt, s->sc, sp, n, X, Y, dD, de, dT);
  cudaError_t e = cudaGetLastError();
  const int blocks = (int)std::min<long long>(s->num_sms * 4, (n + surr::kGateThreads - 1) / surr::kGateThreads);
  cudaEvent_t ev[4];
  for (auto& x : ev) cudaEventCreate(&x);
  for (int mode = 0; mode < 2 && e == cudaSuccess; ++mode) {
    for (int w = 0; w < 2; ++w)
      surr::k_gated<<<blocks, surr::kGateThreads, sizeof(surr::GateSmem), s->stream>>>(
          s->wbf, s->params, s->mt, s->sc, (float)gate_tol, mode, n, dD, de, dT, dFo, ddep, dtau, nullptr, nullptr);
    cudaMemsetAsync(dc, 0, sizeof(surr::GateOut), s->stream);
    cudaEventRecord(ev[2 * mode], s->stream);
    for (int it = 0; it < iters; ++it)
      surr::k_gated<<<blocks, surr::kGateThreads, sizeof(surr::GateSmem), s->stream>>>(
          s->wbf, s->params, s->mt, s->sc, (float)gate_tol, mode, n, dD, de, dT, dFo, ddep, dtau, nullptr,
          it == 0 ? dc : nullptr);
    cudaEventRecord(ev[2 * mode + 1], s->stream);
    e = cudaGetLastError();
  }
  surr::GateOut hc{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hc, dc, sizeof hc, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  float t0 = 0, t1 = 0;
  if (e == cudaSuccess) {
    cudaEventElapsedTime(&t0, ev[0], ev[1]);
    cudaEventElapsedTime(&t1, ev[2], ev[3]);
  }
  for (auto& x : ev) cudaEventDestroy(x);
  void* bufs[] = {X, Y, dD, de, dT, dFo, ddep, dtau, dc};
  for (void* b : bufs) cudaFree(b);
  if (e != cudaSuccess) return sfail(s, MPM_ERR_CUDA, cudaGetErrorString(e));
  *ms_exact = t0 / iters;
  *ms_learned = t1 / iters;
  if (counts) {
    counts->elastic = hc.elastic;
    counts->learned = hc.learned;
    counts->fallback = hc.fallback;
  }
  return MPM_OK;
}

}  // extern "C"
