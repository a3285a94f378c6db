// The learned return map's network (8 -> 64 -> 64 -> 7, ReLU): parameter layout, BF16 tensor-core
// copies and the warp-level forward pass, shared by the surrogate kernels (surrogate.cu) and the
// fused particle pass that runs the network per particle in learned return mode (mpm_kernels.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "mpm_b200.h"

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

static __device__ __forceinline__ float warp_predict_core(const WeightsBf16* w, const float* params, float x0, float x1,
                                                          float x2, float x3, float x4, float x5, float x6, float x7);

// Warp-collective prediction inside a per-particle kernel: every lane of the warp calls it (the
// tensor-core tiles are warp-wide). Lanes with need set get the network's first output for their
// eight inputs x; the others get 0. No lane needs: no tensor-core work. The 32 lanes run as two
// 16-row tiles; the inputs reach the A fragments by shuffles and the output of row r reaches lane r
// the same way. Weights and biases are read through the L1 cache from global memory.
__device__ __forceinline__ float warp_predict_first(const WeightsBf16* w, const float* params, const float x[8],
                                                    bool need) {
  if (!__any_sync(0xffffffffu, need)) return 0.f;
  return warp_predict_core(w, params, x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7]);
}

// The forward pass of one 16-row tile with few registers live, for kernels that hold a particle's
// state around it: the hidden activations are packed to BF16 A fragments as soon as they are formed, and the
// second layer is produced two column tiles at a time, each pair feeding the output layer at once.
__device__ __forceinline__ void forward_lean1(const WeightsBf16& w, const float* bias, const uint32_t xa[4], float y[4],
                                             int g, int tig) {
  uint32_t a1[4][4];  // layer-1 activations as the layer-2 A fragments (K chunks of 16)
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    float h[2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int nt = 2 * kc + u;
      const float b0 = bias[kB1 + nt * 8 + tig * 2], b1 = bias[kB1 + nt * 8 + tig * 2 + 1];
      h[u][0] = b0; h[u][1] = b1; h[u][2] = b0; h[u][3] = b1;
      const __nv_bfloat16* wr = w.w1f + (nt * 8 + g) * 16 + tig * 2;
      mma(h[u], xa, ld32(wr), ld32(wr + 8));
#pragma unroll
      for (int j = 0; j < 4; ++j) h[u][j] = fmaxf(h[u][j], 0.f);
    }
    chain(h, 0, a1[kc]);
  }
  {
    const float b0 = bias[kB3 + tig * 2], b1 = bias[kB3 + tig * 2 + 1];
    y[0] = b0; y[1] = b1; y[2] = b0; y[3] = b1;
  }
#pragma unroll
  for (int oc = 0; oc < 4; ++oc) {  // layer-2 column tiles 2 oc, 2 oc + 1 = layer-3 K chunk oc
    float h[2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int nt = 2 * oc + u;
      const float b0 = bias[kB2 + nt * 8 + tig * 2], b1 = bias[kB2 + nt * 8 + tig * 2 + 1];
      h[u][0] = b0; h[u][1] = b1; h[u][2] = b0; h[u][3] = b1;
#pragma unroll
      for (int kc = 0; kc < 4; ++kc) {
        const __nv_bfloat16* wr = w.w2f + (nt * 8 + g) * kHid + kc * 16 + tig * 2;
        mma(h[u], a1[kc], ld32(wr), ld32(wr + 8));
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) h[u][j] = fmaxf(h[u][j], 0.f);
    }
    uint32_t a[4];
    chain(h, 0, a);
    const __nv_bfloat16* wr = w.w3f + g * kHid + oc * 16 + tig * 2;
    mma(y, a, ld32(wr), ld32(wr + 8));
  }
}

// The forward pass of a warp's two 16-row tiles with few registers live, for kernels that hold a
// particle's state around it: the hidden activations are packed to BF16 A fragments as soon as they
// are formed, the second layer is produced two column tiles at a time, each pair feeding the output
// layer at once, and each B fragment (weights) is loaded once for both tiles, whose MMA chains
// interleave.
__device__ __forceinline__ void forward_lean(const WeightsBf16& w, const float* bias, const uint32_t xa[2][4],
                                              float y[2][4], int g, int tig) {
  uint32_t a1[2][4][4];  // per tile: layer-1 activations as the layer-2 A fragments
#pragma unroll
  for (int kc = 0; kc < 4; ++kc) {
    float h[2][2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int nt = 2 * kc + u;
      const float b0 = bias[kB1 + nt * 8 + tig * 2], b1 = bias[kB1 + nt * 8 + tig * 2 + 1];
      const __nv_bfloat16* wr = w.w1f + (nt * 8 + g) * 16 + tig * 2;
      const uint32_t w0 = ld32(wr), w1 = ld32(wr + 8);
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        h[t][u][0] = b0; h[t][u][1] = b1; h[t][u][2] = b0; h[t][u][3] = b1;
        mma(h[t][u], xa[t], w0, w1);
#pragma unroll
        for (int j = 0; j < 4; ++j) h[t][u][j] = fmaxf(h[t][u][j], 0.f);
      }
    }
#pragma unroll
    for (int t = 0; t < 2; ++t) chain(h[t], 0, a1[t][kc]);
  }
  {
    const float b0 = bias[kB3 + tig * 2], b1 = bias[kB3 + tig * 2 + 1];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      y[t][0] = b0; y[t][1] = b1; y[t][2] = b0; y[t][3] = b1;
    }
  }
#pragma unroll
  for (int oc = 0; oc < 4; ++oc) {  // layer-2 column tiles 2 oc, 2 oc + 1 = layer-3 K chunk oc
    float h[2][2][4];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int nt = 2 * oc + u;
      const float b0 = bias[kB2 + nt * 8 + tig * 2], b1 = bias[kB2 + nt * 8 + tig * 2 + 1];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        h[t][u][0] = b0; h[t][u][1] = b1; h[t][u][2] = b0; h[t][u][3] = b1;
      }
#pragma unroll
      for (int kc = 0; kc < 4; ++kc) {
        const __nv_bfloat16* wr = w.w2f + (nt * 8 + g) * kHid + kc * 16 + tig * 2;
        const uint32_t w0 = ld32(wr), w1 = ld32(wr + 8);
#pragma unroll
        for (int t = 0; t < 2; ++t) mma(h[t][u], a1[t][kc], w0, w1);
      }
#pragma unroll
      for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int j = 0; j < 4; ++j) h[t][u][j] = fmaxf(h[t][u][j], 0.f);
    }
    const __nv_bfloat16* wr = w.w3f + g * kHid + oc * 16 + tig * 2;
    const uint32_t w0 = ld32(wr), w1 = ld32(wr + 8);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      uint32_t a[4];
      chain(h[t], 0, a);
      mma(y[t], a, w0, w1);
    }
  }
}

static __device__ __forceinline__ float warp_predict_core(const WeightsBf16* w, const float* params, float x0, float x1,
                                                          float x2, float x3, float x4, float x5, float x6, float x7) {
  const float x[8] = {x0, x1, x2, x3, x4, x5, x6, x7};
  __syncwarp();
  const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  uint32_t xa[2][4];
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const int r0 = half * 16 + g, r1 = r0 + 8;
    // inputs 2 tig, 2 tig + 1 of rows r0 and r1 (columns 8..15 of K are zero)
    float a00 = 0.f, a01 = 0.f, a10 = 0.f, a11 = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float p0 = __shfl_sync(0xffffffffu, x[2 * j], r0), p1 = __shfl_sync(0xffffffffu, x[2 * j + 1], r0);
      const float q0 = __shfl_sync(0xffffffffu, x[2 * j], r1), q1 = __shfl_sync(0xffffffffu, x[2 * j + 1], r1);
      if (tig == j) {
        a00 = p0; a01 = p1; a10 = q0; a11 = q1;
      }
    }
    xa[half][0] = pack_bf16(a00, a01);
    xa[half][1] = pack_bf16(a10, a11);
    xa[half][2] = 0u;
    xa[half][3] = 0u;
  }
  float y[2][4];
  forward_lean(*w, params, xa, y, g, tig);
  // output column 0 of row r of a tile sits in lane 4 (r % 8): y[0] for r < 8, y[2] for r >= 8
  const int r = lane & 15, src = 4 * (r & 7);
  float out = 0.f;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const float lo = __shfl_sync(0xffffffffu, y[half][0], src), hi = __shfl_sync(0xffffffffu, y[half][2], src);
    if ((lane >> 4) == half) out = r < 8 ? lo : hi;
  }
  return out;
}

// warp_predict_core with the warp's two tiles one after the other (forward_lean1): fewer registers
// live, for the fused particle pass, where the network branch shares the 128 registers of a thread
// with the particle's state (2% less pass time than the two-tile form there).
static __device__ __forceinline__ float warp_predict_seq(const WeightsBf16* w, const float* params, float x0, float x1,
                                                         float x2, float x3, float x4, float x5, float x6, float x7) {
  const float x[8] = {x0, x1, x2, x3, x4, x5, x6, x7};
  __syncwarp();
  const int lane = threadIdx.x & 31, g = lane >> 2, tig = lane & 3;
  float out = 0.f;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const int r0 = half * 16 + g, r1 = r0 + 8;
    // inputs 2 tig, 2 tig + 1 of rows r0 and r1 (columns 8..15 of K are zero)
    float a00 = 0.f, a01 = 0.f, a10 = 0.f, a11 = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float p0 = __shfl_sync(0xffffffffu, x[2 * j], r0), p1 = __shfl_sync(0xffffffffu, x[2 * j + 1], r0);
      const float q0 = __shfl_sync(0xffffffffu, x[2 * j], r1), q1 = __shfl_sync(0xffffffffu, x[2 * j + 1], r1);
      if (tig == j) {
        a00 = p0; a01 = p1; a10 = q0; a11 = q1;
      }
    }
    const uint32_t xa[4] = {pack_bf16(a00, a01), pack_bf16(a10, a11), 0u, 0u};
    float y[4];
    forward_lean1(*w, params, xa, y, g, tig);
    // output column 0 of row r sits in lane 4 (r % 8): y[0] for r < 8, y[2] for r >= 8
    const int r = lane - half * 16;
    const int src = 4 * (r & 7);
    const float lo = __shfl_sync(0xffffffffu, y[0], src), hi = __shfl_sync(0xffffffffu, y[2], src);
    if (r >= 0 && r < 16) out = r < 8 ? lo : hi;
  }
  return out;
}

// Host side (surrogate.cu): the material model a network was made for, and a copy of its BF16
// weights (weights_bytes() bytes at dst_w) and FP32 parameters (kParams floats) into device memory
// owned by the caller, ordered on stream st.
int surrogate_model(const mpm_surrogate* s);
size_t weights_bytes();
int export_weights(mpm_surrogate* s, void* dst_w, float* dst_params, cudaStream_t st);

}  // namespace surr
