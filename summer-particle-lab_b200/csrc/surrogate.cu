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
// Arithmetic. Weights and activations enter the tensor cores as BF16 with FP32 accumulation; the
// optimizer keeps FP32 master weights. Training (k_train_tc) and the gated map over particle arrays
// (k_gated) run on the 5th-generation tensor cores: tcgen05.mma with operands in shared memory and
// accumulators in tensor memory, 128 samples per tile, the weight gradients as GEMMs over the
// sample axis accumulated in tensor memory. The per-particle inference inside other kernels
// (k_gated_jc, the fused particle pass in learned return mode) runs warp-wide mma.sync tiles of 16
// rows, where the accumulator fragment of one layer is the A fragment of the next, so activations
// never leave registers.
//
// Johnson-Cook (models 6, 7). The network maps the dimensionless trial state to the root of the
// consistency condition the reference bisects (see k_samples_jc); mpm::jc_refine polishes the
// prediction by Newton steps and gates it on the consistency residual.
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
#include "mpm_internal.h"
#include "mpm_math.h"
#include "surrogate_net.h"

namespace surr {

__device__ __forceinline__ void load_weights(WeightsBf16& dst, const WeightsBf16* src) {
  const uint4* s = reinterpret_cast<const uint4*>(src);
  uint4* d = reinterpret_cast<uint4*>(&dst);
  for (int i = threadIdx.x; i < (int)(sizeof(WeightsBf16) / 16); i += blockDim.x) d[i] = s[i];
}

// ---------------------------------------------------------------------------------------------
// Training step on the 5th-generation tensor cores (tcgen05, accumulators in tensor memory).
//
// One CTA of 4 warps per SM takes tiles of 128 samples (the MMA's M); tile row r is thread r and
// TMEM lane r. Every GEMM of the step is one chain of tcgen05.mma (kind::f16, BF16 operands in
// shared memory, FP32 accumulation in TMEM) issued by thread 0 and completed through an mbarrier:
//   forward   H1 = X W1^T, H2 = relu(H1) W2^T, Y = relu(H2) W3^T
//   backward  dH2 = dY W3, dH1 = (dH2 . relu'(H2)) W2
//   weights   [dW2 ; dW1] += [d2^T ; d1^T] [h1^T | x^T | 1]^T  (M = 128: o of layer 2, then of layer 1)
//             dW3 += dy^T [h2^T | 1]^T, whose columns of ones give the bias gradients.
// Between the GEMMs the threads read their accumulator row (tcgen05.ld), apply bias, ReLU, loss or
// mask, and write the next operands to shared memory in the canonical K-major layout without
// swizzle (8 x 8 core matrices of 128 bytes; an 8-row group holds its K chunks back to back), both
// as rows (A of the next layer) and transposed (the sample axis as K of the weight GEMMs). The
// weight-gradient accumulators stay in TMEM across the CTA's tiles and leave once per CTA.

constexpr int kTcRows = 128;
constexpr int kTcThreads = 128;
constexpr int kTmemCols = 512;
// accumulator columns (32-bit) in the CTA's tensor memory
constexpr int kColH1 = 0, kColH2 = 64, kColY = 128, kColD2 = 144, kColD1 = 208, kColW21 = 272, kColW3 = 368;

struct __align__(1024) TcSmem {
  __nv_bfloat16 w1[64 * 16];    // B of H1:  [N 64 outputs][K 16 inputs]
  __nv_bfloat16 w2[64 * 64];    // B of H2:  [64][64]
  __nv_bfloat16 w3[16 * 64];    // B of Y:   [N 16][K 64] (rows 7..15 zero)
  __nv_bfloat16 w3t[64 * 16];   // B of dH2: [N 64][K 16] (W3 transposed, K 7..15 zero)
  __nv_bfloat16 w2t[64 * 64];   // B of dH1: [N 64][K 64] (W2 transposed)
  __nv_bfloat16 x[128 * 16];    // A: inputs (columns 8..15 zero)
  __nv_bfloat16 h1[128 * 64];   // A: layer-1 activations
  __nv_bfloat16 h2[128 * 64];   // A: layer-2 activations
  __nv_bfloat16 dy[128 * 16];   // A: output gradient (columns 7..15 zero)
  __nv_bfloat16 d2[128 * 64];   // A: layer-2 pre-activation gradient
  __nv_bfloat16 dyT[16 * 128];  // A of dW3; as an M = 128 operand its rows 16..127 run into dT (not read back)
  __nv_bfloat16 dT[128 * 128];  // A of [dW2; dW1]: rows 0..63 d2^T, rows 64..127 d1^T (K = samples)
  __nv_bfloat16 hxT[96 * 128];  // B of [dW2; dW1]: rows 0..63 h1^T, 64..79 x^T, 80 ones, 81..95 zero
  __nv_bfloat16 h2T[80 * 128];  // B of dW3: rows 0..63 h2^T, 64 ones, 65..79 zero
  float bias[64 + 64 + 16];
  unsigned long long mbar;
  unsigned tmem_base;
};

// Element offset of (row r, column k) in a K-major no-swizzle bf16 matrix with K columns.
__device__ __forceinline__ int km_off(int r, int k, int K) { return (r & 7) * 8 + (r >> 3) * (K * 8) + (k & 7) + (k >> 3) * 64; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Shared-memory matrix descriptor of K-major operand rows (K columns) for the MMA's K step ks
// (16 columns): start, leading byte offset 128 (the next 8 columns), stride byte offset 16 K (the
// next 8 rows), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t kdesc(const void* base, int K, int ks) {
  const uint32_t a = smem_u32(base) + ks * 256;
  return static_cast<uint64_t>((a >> 4) & 0x3FFFu) | (static_cast<uint64_t>(128 >> 4) << 16) |
         (static_cast<uint64_t>((K * 16) >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor: kind::f16, BF16 A and B (K-major), FP32 D, M = 128, N.
__device__ __forceinline__ uint32_t idesc_bf16(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

// D (+)= A B^T over K columns (A: 128 rows, B: N rows, both K-major).
__device__ __forceinline__ void tc_gemm(uint32_t d_tmem, const void* A, const void* B, int K, int N, bool accumulate) {
  const uint32_t id = idesc_bf16(N);
  for (int ks = 0; ks < K / 16; ++ks) umma_f16(d_tmem, kdesc(A, K, ks), kdesc(B, K, ks), id, (accumulate || ks > 0) ? 1u : 0u);
}

__device__ __forceinline__ void tc_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Waits for the mbarrier phase with the given parity for at most 2^31 SM cycles (about 1 s); false
// if it gave up.
__device__ __forceinline__ bool tc_wait(unsigned long long* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const long long t0 = clock64();
  while (clock64() - t0 < (1ll << 31)) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void st_pair(__nv_bfloat16* m, int off, float a, float b) {
  *reinterpret_cast<uint32_t*>(m + off) = pack_bf16(a, b);
}

// Operands written by this CTA's threads become visible to the tensor cores before thread 0 issues.
__device__ __forceinline__ void tc_handoff() {
  proxy_fence();
  tc_fence_before();
  __syncthreads();
}

// One MMA group: thread 0 issues it after the hand-off and commits it to the mbarrier, every thread
// waits for its completion (bounded). Returns false for the whole CTA if a wait gave up.
template <typename Issue>
__device__ __forceinline__ bool tc_run(unsigned long long* bar, uint32_t& phase, Issue issue) {
  tc_handoff();
  if (threadIdx.x == 0) {
    tc_fence_after();
    issue();
    tc_commit(bar);
  }
  const bool done = tc_wait(bar, phase);
  phase ^= 1u;
  tc_fence_after();
  return __syncthreads_and(done) != 0;
}

__device__ __forceinline__ void tc_alloc(unsigned* dst, int cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_dealloc(uint32_t taddr, int cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

__device__ __forceinline__ void mbar_init1(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Loss = sum over samples and outputs of wout[o] ws (y - t)^2 / batch, with ws = Y[row][7] the
// sample weight; its gradient is added to grad_out and the loss to loss_out. Sample r of this call
// is row (first + r * stride) mod n_data, a strided walk that visits every row once per epoch when
// stride and n_data are coprime. err: set when a completion wait gave up.
__global__ void __launch_bounds__(kTcThreads, 1)
    k_train_tc(const WeightsBf16* wg, const float* params, const float* X, const float* Y, long long n_data,
               long long first, long long stride, int batch, float inv_batch, const float* wout, float* grad_out,
               float* loss_out, unsigned* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  TcSmem& sm = *reinterpret_cast<TcSmem*>(smem_raw);
  const int r = threadIdx.x, warp = r >> 5;
  // weights into the K-major layouts, constant rows, biases
  for (int i = r; i < 64 * 16; i += kTcThreads) {
    const int o = i / 16, k = i % 16;
    sm.w1[km_off(o, k, 16)] = wg->w1f[o * 16 + k];
    sm.w3t[km_off(o, k, 16)] = wg->w3b[o * 16 + k];  // w3b is [i][o], o padded to 16
  }
  for (int i = r; i < 64 * 64; i += kTcThreads) {
    const int o = i / 64, k = i % 64;
    sm.w2[km_off(o, k, 64)] = wg->w2f[i];
    sm.w2t[km_off(o, k, 64)] = wg->w2b[i];
  }
  for (int i = r; i < 16 * 64; i += kTcThreads) {
    const int o = i / 64, k = i % 64;
    sm.w3[km_off(o, k, 64)] = o < 8 ? wg->w3f[o * 64 + k] : __float2bfloat16_rn(0.f);
  }
  for (int i = r; i < 144; i += kTcThreads)
    sm.bias[i] = i < 64 ? params[kB1 + i] : i < 128 ? params[kB2 + i - 64] : (i - 128 < 8 ? params[kB3 + i - 128] : 0.f);
  for (int n = 72; n < 96; ++n) sm.hxT[km_off(n, r, 128)] = __float2bfloat16_rn(n == 80 ? 1.f : 0.f);
  for (int n = 64; n < 80; ++n) sm.h2T[km_off(n, r, 128)] = __float2bfloat16_rn(n == 64 ? 1.f : 0.f);
  if (r == 0) mbar_init1(&sm.mbar);
  if (warp == 0) tc_alloc(&sm.tmem_base, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = sm.tmem_base;
  const uint32_t lane = static_cast<uint32_t>(warp * 32) << 16;  // this warp's TMEM lane quarter
  float wo[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) wo[k] = k < 7 ? wout[k] : 0.f;
  uint32_t phase = 0;
  float loss = 0.f;
  int ntile = 0;
  bool ok = true;
  const int tiles = (batch + kTcRows - 1) / kTcRows;
  for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++ntile) {
    const int srow = tile * kTcRows + r;
    const bool valid = srow < batch;
    const long long row = valid ? (first + static_cast<long long>(srow) * stride) % n_data : 0;
    float xv[8], tv[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      xv[k] = valid ? X[row * 8 + k] : 0.f;
      tv[k] = valid ? Y[row * 8 + k] : 0.f;
    }
    const float ws = tv[7];  // sample weight (0 for the rows past the batch)
#pragma unroll
    for (int k = 0; k < 16; k += 2) st_pair(sm.x, km_off(r, k, 16), k < 8 ? xv[k] : 0.f, k < 8 ? xv[k + 1] : 0.f);
#pragma unroll
    for (int k = 0; k < 8; ++k) sm.hxT[km_off(64 + k, r, 128)] = __float2bfloat16_rn(xv[k]);
    // layer 1
    ok = tc_run(&sm.mbar, phase, [&] { tc_gemm(tm + kColH1, sm.x, sm.w1, 16, 64, false); });
    if (!ok) break;
    uint32_t m1[2] = {0u, 0u}, m2[2] = {0u, 0u};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tmem_ld16(tm + lane + kColH1 + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; j += 2) {
        const int o = 16 * c + j;
        const float a = fmaxf(v[j] + sm.bias[o], 0.f), b = fmaxf(v[j + 1] + sm.bias[o + 1], 0.f);
        m1[o >> 5] |= (a > 0.f ? 1u : 0u) << (o & 31);
        m1[(o + 1) >> 5] |= (b > 0.f ? 1u : 0u) << ((o + 1) & 31);
        st_pair(sm.h1, km_off(r, o, 64), a, b);
        sm.hxT[km_off(o, r, 128)] = __float2bfloat16_rn(a);
        sm.hxT[km_off(o + 1, r, 128)] = __float2bfloat16_rn(b);
      }
    }
    // layer 2
    ok = tc_run(&sm.mbar, phase, [&] { tc_gemm(tm + kColH2, sm.h1, sm.w2, 64, 64, false); });
    if (!ok) break;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tmem_ld16(tm + lane + kColH2 + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; j += 2) {
        const int o = 16 * c + j;
        const float a = fmaxf(v[j] + sm.bias[64 + o], 0.f), b = fmaxf(v[j + 1] + sm.bias[64 + o + 1], 0.f);
        m2[o >> 5] |= (a > 0.f ? 1u : 0u) << (o & 31);
        m2[(o + 1) >> 5] |= (b > 0.f ? 1u : 0u) << ((o + 1) & 31);
        st_pair(sm.h2, km_off(r, o, 64), a, b);
        sm.h2T[km_off(o, r, 128)] = __float2bfloat16_rn(a);
        sm.h2T[km_off(o + 1, r, 128)] = __float2bfloat16_rn(b);
      }
    }
    // output layer, loss and dL/dy = 2 w (y - t) / batch (output 7 is padding)
    ok = tc_run(&sm.mbar, phase, [&] { tc_gemm(tm + kColY, sm.h2, sm.w3, 64, 16, false); });
    if (!ok) break;
    {
      float v[16];
      tmem_ld16(tm + lane + kColY, v);
      float dy[16];
#pragma unroll
      for (int o = 0; o < 16; ++o) {
        const float e = o < 7 ? v[o] + sm.bias[128 + o] - tv[o] : 0.f;
        dy[o] = 2.f * wo[o & 7] * ws * e * inv_batch;
        loss += ws * wo[o & 7] * e * e * inv_batch;
      }
#pragma unroll
      for (int o = 0; o < 16; o += 2) {
        st_pair(sm.dy, km_off(r, o, 16), dy[o], dy[o + 1]);
        sm.dyT[km_off(o, r, 128)] = __float2bfloat16_rn(dy[o]);
        sm.dyT[km_off(o + 1, r, 128)] = __float2bfloat16_rn(dy[o + 1]);
      }
    }
    // dH2 = dY W3 and dW3 += dy^T [h2 | 1]
    const bool acc_w = ntile > 0;
    ok = tc_run(&sm.mbar, phase, [&] {
      tc_gemm(tm + kColD2, sm.dy, sm.w3t, 16, 64, false);
      tc_gemm(tm + kColW3, sm.dyT, sm.h2T, 128, 80, acc_w);
    });
    if (!ok) break;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tmem_ld16(tm + lane + kColD2 + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; j += 2) {
        const int o = 16 * c + j;
        const float a = (m2[o >> 5] >> (o & 31)) & 1u ? v[j] : 0.f;
        const float b = (m2[(o + 1) >> 5] >> ((o + 1) & 31)) & 1u ? v[j + 1] : 0.f;
        st_pair(sm.d2, km_off(r, o, 64), a, b);
        sm.dT[km_off(o, r, 128)] = __float2bfloat16_rn(a);
        sm.dT[km_off(o + 1, r, 128)] = __float2bfloat16_rn(b);
      }
    }
    // dH1 = d2 W2
    ok = tc_run(&sm.mbar, phase, [&] { tc_gemm(tm + kColD1, sm.d2, sm.w2t, 64, 64, false); });
    if (!ok) break;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tmem_ld16(tm + lane + kColD1 + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int o = 16 * c + j;
        sm.dT[km_off(64 + o, r, 128)] = __float2bfloat16_rn((m1[o >> 5] >> (o & 31)) & 1u ? v[j] : 0.f);
      }
    }
    // [dW2; dW1] += [d2^T; d1^T] [h1 | x | 1]
    ok = tc_run(&sm.mbar, phase, [&] { tc_gemm(tm + kColW21, sm.dT, sm.hxT, 128, 96, acc_w); });
  }
  if (ok && ntile > 0) {
    // gradient accumulators out of TMEM, one global add per entry and CTA
#pragma unroll 1
    for (int c = 0; c < 6; ++c) {
      float v[16];
      tmem_ld16(tm + lane + kColW21 + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = 16 * c + j;
        if (r < 64) {  // layer 2, output r
          if (n < 64) atomicAdd(&grad_out[kW2 + r * 64 + n], v[j]);
          else if (n == 80) atomicAdd(&grad_out[kB2 + r], v[j]);
        } else {  // layer 1, output r - 64
          if (n >= 64 && n < 72) atomicAdd(&grad_out[kW1 + (r - 64) * 16 + (n - 64)], v[j]);
          else if (n == 80) atomicAdd(&grad_out[kB1 + (r - 64)], v[j]);
        }
      }
    }
#pragma unroll 1
    for (int c = 0; c < 5; ++c) {
      float v[16];
      tmem_ld16(tm + lane + kColW3 + 16 * c, v);
      if (r < kOut) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = 16 * c + j;
          if (n < 64) atomicAdd(&grad_out[kW3 + r * 64 + n], v[j]);
          else if (n == 64) atomicAdd(&grad_out[kB3 + r], v[j]);
        }
      }
    }
  }
  if (!ok) {
    // a completion wait gave up: one more bounded wait for the MMA group in flight, then leave
    tc_wait(&sm.mbar, phase);
    if (r == 0) atomicOr(err, 1u);
  }
  for (int o = 16; o; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if ((r & 31) == 0 && loss != 0.f) atomicAdd(loss_out, loss);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tc_dealloc(tm, kTmemCols);
  }
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
  float dt_lo, dt_hi;          // log-uniform substep (rate-dependent laws)
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
// Gated return map over particles, 128 per tile: thread r owns particle r of the tile and TMEM lane
// r; when a tile holds a plastic particle the network runs as three tcgen05 GEMMs (M = 128) with
// the epilogues of k_train_tc's forward pass.
constexpr int kGateThreads = 128;
constexpr int kGateTmemCols = 128;  // H1 and then H2 in columns 0..63 (H1 is read before H2 lands), Y 64..79

struct __align__(1024) GateSmem {
  __nv_bfloat16 w1[64 * 16];
  __nv_bfloat16 w2[64 * 64];
  __nv_bfloat16 w3[16 * 64];
  __nv_bfloat16 x[128 * 16];
  __nv_bfloat16 h1[128 * 64];
  __nv_bfloat16 h2[128 * 64];
  float bias[64 + 64 + 16];
  unsigned long long mbar;
  unsigned tmem_base;
};

struct GateOut {
  unsigned elastic, learned, fallback;
};

// Stages the BF16 weights in the canonical layouts and the biases, initialises the completion
// barrier and allocates the tile's TMEM columns; returns their base. Every thread of the CTA calls it.
__device__ __forceinline__ uint32_t gate_setup(GateSmem& sm, const WeightsBf16* wg, const float* params) {
  const int r = threadIdx.x, warp = r >> 5;
  for (int i = r; i < 64 * 16; i += kGateThreads) sm.w1[km_off(i / 16, i % 16, 16)] = wg->w1f[i];
  for (int i = r; i < 64 * 64; i += kGateThreads) sm.w2[km_off(i / 64, i % 64, 64)] = wg->w2f[i];
  for (int i = r; i < 16 * 64; i += kGateThreads)
    sm.w3[km_off(i / 64, i % 64, 64)] = i / 64 < 8 ? wg->w3f[i] : __float2bfloat16_rn(0.f);
  for (int i = r; i < 144; i += kGateThreads)
    sm.bias[i] = i < 64 ? params[kB1 + i] : i < 128 ? params[kB2 + i - 64] : (i - 128 < 8 ? params[kB3 + i - 128] : 0.f);
  if (r == 0) mbar_init1(&sm.mbar);
  if (warp == 0) tc_alloc(&sm.tmem_base, kGateTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  return sm.tmem_base;
}

// The network on the tile's 128 input rows (thread r writes row r, x[8]): three tcgen05 GEMM groups
// (M = 128) with the ReLU epilogues of k_train_tc's forward pass; y[0..6] are thread r's outputs
// before the output bias (y[7..15] are zero). Returns false when a completion wait gave up (the
// tile's outputs are then not to be used). Every thread of the CTA calls it.
__device__ __forceinline__ bool gate_network(GateSmem& sm, uint32_t tm, uint32_t& phase, const float x[8], float y[16]) {
  const int r = threadIdx.x;
  const uint32_t lane = static_cast<uint32_t>((r >> 5) * 32) << 16;
#pragma unroll
  for (int k = 0; k < 16; k += 2) st_pair(sm.x, km_off(r, k, 16), k < 8 ? x[k] : 0.f, k < 8 ? x[k + 1] : 0.f);
  bool ok = tc_run(&sm.mbar, phase, [&] { tc_gemm(tm + 0, sm.x, sm.w1, 16, 64, false); });
  if (ok) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tmem_ld16(tm + lane + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; j += 2)
        st_pair(sm.h1, km_off(r, 16 * c + j, 64), fmaxf(v[j] + sm.bias[16 * c + j], 0.f),
                fmaxf(v[j + 1] + sm.bias[16 * c + j + 1], 0.f));
    }
    ok = tc_run(&sm.mbar, phase, [&] { tc_gemm(tm + 0, sm.h1, sm.w2, 64, 64, false); });
  }
  if (ok) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      float v[16];
      tmem_ld16(tm + lane + 16 * c, v);
#pragma unroll
      for (int j = 0; j < 16; j += 2)
        st_pair(sm.h2, km_off(r, 16 * c + j, 64), fmaxf(v[j] + sm.bias[64 + 16 * c + j], 0.f),
                fmaxf(v[j + 1] + sm.bias[64 + 16 * c + j + 1], 0.f));
    }
    ok = tc_run(&sm.mbar, phase, [&] { tc_gemm(tm + 64, sm.h2, sm.w3, 64, 16, false); });
  }
  if (ok) tmem_ld16(tm + lane + 64, y);
  return ok;
}

// Releases the TMEM columns (after one more bounded wait when a group may still be in flight).
__device__ __forceinline__ void gate_teardown(GateSmem& sm, uint32_t tm, uint32_t phase, bool tc_ok) {
  if (!tc_ok) tc_wait(&sm.mbar, phase);
  tc_fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) {
    tc_fence_after();
    tc_dealloc(tm, kGateTmemCols);
  }
}

// D = F - I (n x 9 float, formed by the caller in higher precision), ep, T in; D, dep and tau
// (n x 6: xx yy zz xy xz yz) out; path: 0 elastic, 1 learned, 2 exact fallback. use_mlp = 0 runs
// the exact map for every particle through the same kernel, so both timings share loads and stores.
// err: set when a tensor-core completion wait gave up (the tile's predictions are then rejected).
__global__ void __launch_bounds__(kGateThreads) k_gated(const WeightsBf16* wg, const float* params, mpm::MaterialDev mt,
                                                        Scales sc, float gate_tol, int use_mlp, long long n,
                                                        const float* Din, const float* epin, const float* Tin, float* Dout,
                                                        float* dep, float* tau, signed char* path, GateOut* counts,
                                                        unsigned* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  GateSmem& sm = *reinterpret_cast<GateSmem*>(smem_raw);
  const int r = threadIdx.x;
  uint32_t tm = 0, phase = 0;
  bool tc_ok = true;
  if (use_mlp) tm = gate_setup(sm, wg, params);
  unsigned c_el = 0, c_ml = 0, c_fb = 0;
  const float r2 = 1.41421356237f, ir2 = 0.70710678118f, s15 = 1.224744871391589f;
  for (long long base = (long long)blockIdx.x * kGateThreads; base < n; base += (long long)gridDim.x * kGateThreads) {
    const long long i = base + r;
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
    if (use_mlp && tc_ok && __syncthreads_or(plastic)) {
      float x[8];
      features(sc, tr, T, ep, x);
      float y[16];
      tc_ok = gate_network(sm, tm, phase, x, y);
      if (tc_ok) {
#pragma unroll
        for (int k = 0; k < 7; ++k) y[k] += sm.bias[128 + k];
      } else if (r == 0) {
        atomicOr(err, 1u);
      }
      if (plastic && tc_ok) {
        float t6[6];
        trial_stress(mt, L6, t6);
        const float smag = 2.f * mt.mu * s15 * tr.dep_est;
        for (int k = 0; k < 6; ++k) tau6[k] = t6[k] + smag * y[k];
        dp = tr.dep_est * y[6];
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
      if (accepted) {
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
        // elastic states and the exact fallback share one call (the return only where plastic),
        // so a warp holding both runs the constitutive update once
        const mpm::ConstitutiveOut co = mpm::constitutive_update(mt, D, ep, T, 0.f, plastic);
        tau6[0] = co.tau.xx; tau6[1] = co.tau.yy; tau6[2] = co.tau.zz;
        tau6[3] = co.tau.xy * r2; tau6[4] = co.tau.xz * r2; tau6[5] = co.tau.yz * r2;
        dp = plastic ? co.dep : 0.f;
        if (plastic) ++c_fb; else ++c_el;
        if (path) path[i] = plastic ? 2 : 0;
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
    if ((r & 31) == 0) {
      atomicAdd(&counts->elastic, c_el);
      atomicAdd(&counts->learned, c_ml);
      atomicAdd(&counts->fallback, c_fb);
    }
  }
  if (use_mlp) gate_teardown(sm, tm, phase, tc_ok);
}

// ---------------------------------------------------------------------------------------------
// Johnson-Cook (models 6, 7): the network maps the dimensionless trial state (mpm::jc_features) to
// the consistency root u = dep / s of src/three/metal-plasticity.js:28-34 (output 0); the in-step
// use refines it by Newton steps and gates it (mpm::jc_refine).

// One random Johnson-Cook trial state: tr e uniform in [-0.01, 0.01], ep and T uniform, the substep
// log-uniform; even draws take |dev e| log-uniform, odd draws a trial stress just above the
// initial flow stress, q = flow(ep, 0, T) (1 + d) with d log-uniform in [1e-4, 1] (the states of
// a loading step, whose increment is small).
struct JcState {
  float q, J, ep, T, dt;
};

__device__ JcState jc_random_state(const mpm::MaterialDev& mt, const SampleSpec& sp, long long i) {
  JcState st;
  const float trv = 0.02f * urand(sp.seed, i, 1) - 0.01f;
  st.J = expf(trv);
  st.ep = sp.ep_hi * urand(sp.seed, i, 2);
  st.T = sp.T_lo + (sp.T_hi - sp.T_lo) * urand(sp.seed, i, 3);
  st.dt = expf(logf(sp.dt_lo) + urand(sp.seed, i, 4) * (logf(sp.dt_hi) - logf(sp.dt_lo)));
  if (i & 1) {
    const float d = expf(-9.210340372f * (1.f - urand(sp.seed, i, 0)));
    st.q = mpm::jc_flow(mt, st.ep, 0.f, st.T) * (1.f + d);
  } else {
    const float mag = expf(logf(sp.strain_lo) + urand(sp.seed, i, 0) * (logf(sp.strain_hi) - logf(sp.strain_lo)));
    st.q = 2.449489742783178f * mt.mu * mag / st.J;
  }
  return st;
}

// Training rows for Johnson-Cook: X the eight inputs, Y[0] the exact root u from the bisection,
// Y[7] the sample weight (1 for plastic states; elastic states have no return and weight 0).
__global__ void k_samples_jc(mpm::MaterialDev mt, SampleSpec sp, long long n, float* X, float* Y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const JcState st = jc_random_state(mt, sp, i);
    const bool plastic = st.q > mpm::jc_flow(mt, st.ep, 0.f, st.T);
    float x[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float u = 0.f;
    if (plastic) {
      mpm::jc_features(mt, st.q, st.J, st.ep, st.T, st.dt, x);
      const float s = st.q * st.J / (3.f * mt.mu);
      u = mpm::jc_bisect(mt, st.q, st.J, st.ep, st.T, st.dt) / s;
    }
    for (int k = 0; k < 8; ++k) X[i * 8 + k] = x[k];
    Y[i * 8 + 0] = u;
    for (int k = 1; k < 7; ++k) Y[i * 8 + k] = 0.f;
    Y[i * 8 + 7] = plastic ? 1.f : 0.f;
  }
}

// The plastic increment of random Johnson-Cook trial states: exact bisection for every state
// (use_mlp 0), or the network (warp-wide tensor-core tiles, use_mlp 1) or the initial flow stress's
// guess (use_mlp 2) + Newton refinement + gate with the bisection for rejected states. dep out
// (keeps the work); counts: elastic, accepted, rejected.
__global__ void __launch_bounds__(256) k_gated_jc(const WeightsBf16* wg, const float* params, mpm::MaterialDev mt,
                                                  SampleSpec sp, float gate_tol, int newton, int use_mlp, long long n,
                                                  float* dep_out, GateOut* counts) {
  unsigned c_el = 0, c_ml = 0, c_fb = 0;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += (long long)gridDim.x * blockDim.x) {
    const long long i = base + threadIdx.x;
    const bool live = i < n;
    const JcState st = jc_random_state(mt, sp, live ? i : 0);
    const bool plastic = live && st.q > mpm::jc_flow(mt, st.ep, 0.f, st.T);
    float dep = 0.f;
    bool accepted = false;
    if (use_mlp == 1) {
      float x[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (plastic) mpm::jc_features(mt, st.q, st.J, st.ep, st.T, st.dt, x);
      const float u = warp_predict_first(wg, params, x, plastic);
      if (plastic) {
        const mpm::JcRefined r = mpm::jc_refine(mt, st.q, st.J, st.ep, st.T, st.dt, u, gate_tol, newton);
        dep = r.dep;
        accepted = r.ok;
      }
    } else if (use_mlp == 2 && plastic) {  // the same refinement from the initial flow stress's guess
      const float u0 = fminf(1.f, fmaxf(0.f, 1.f - mpm::jc_flow(mt, st.ep, 0.f, st.T) / st.q));
      const mpm::JcRefined r = mpm::jc_refine(mt, st.q, st.J, st.ep, st.T, st.dt, u0, gate_tol, newton);
      dep = r.dep;
      accepted = r.ok;
    }
    if (plastic && !accepted) dep = mpm::jc_bisect(mt, st.q, st.J, st.ep, st.T, st.dt);
    if (live) {
      dep_out[i] = dep;
      if (!plastic) ++c_el;
      else if (accepted) ++c_ml;
      else ++c_fb;
    }
  }
  if (counts) {
    for (int o = 16; o; o >>= 1) {
      c_el += __shfl_xor_sync(0xffffffffu, c_el, o);
      c_ml += __shfl_xor_sync(0xffffffffu, c_ml, o);
      c_fb += __shfl_xor_sync(0xffffffffu, c_fb, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&counts->elastic, c_el);
      atomicAdd(&counts->learned, c_ml);
      atomicAdd(&counts->fallback, c_fb);
    }
  }
}

mpm::MaterialDev to_dev(const mpm_material& m) { return mpm::material_to_device(m); }

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
  unsigned* tc_err = nullptr;  // set by a tensor-core kernel when a completion wait gave up
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

surr::SampleSpec spec_of(const mpm_surrogate_config* cfg) {
  surr::SampleSpec sp{(float)cfg->strain_min, (float)cfg->strain_max, (float)cfg->T_min, (float)cfg->T_max,
                      (float)cfg->ep_max, cfg->seed, 1e-7f, 1e-5f};
  if (cfg->dt_min > 0 && cfg->dt_max >= cfg->dt_min) {
    sp.dt_lo = (float)cfg->dt_min;
    sp.dt_hi = (float)cfg->dt_max;
  }
  return sp;
}

bool is_jc(const mpm_surrogate* s) { return mpm::learned_model(s->mat.model); }

// Launch shape of k_gated: with the network, 4 CTAs per SM (128 TMEM columns and 49 KB of shared
// memory each); the exact map alone needs neither, so it runs 16 CTAs per SM for latency hiding.
struct GateLaunch {
  int blocks;
  size_t smem;
};
GateLaunch gate_launch(const mpm_surrogate* s, int use_mlp, long long n) {
  const long long tiles = (n + surr::kGateThreads - 1) / surr::kGateThreads;
  if (use_mlp) return {(int)std::min<long long>(s->num_sms * 4, tiles), sizeof(surr::GateSmem)};
  return {(int)std::min<long long>(s->num_sms * 16, tiles), 0};
}

// One forward/backward pass over `batch` rows (row r of the call is (first + r stride) mod n_data)
// adding the gradient to s->grad and the loss to *loss: tiles of 128 rows, one CTA per SM.
void launch_train(mpm_surrogate* s, const float* X, const float* Y, long long n_data, long long first, long long stride,
                  int batch, const float* wout, float* loss) {
  const int tiles = (batch + surr::kTcRows - 1) / surr::kTcRows;
  const int blocks = std::min(s->num_sms, tiles);
  surr::k_train_tc<<<blocks, surr::kTcThreads, sizeof(surr::TcSmem), s->stream>>>(
      s->wbf, s->params, X, Y, n_data, first, stride, batch, 1.f / batch, wout, s->grad, loss, s->tc_err);
}

// The tensor-core kernels' completion-wait flag (and its clearing).
int check_tc(mpm_surrogate* s) {
  unsigned e = 0;
  if (cudaMemcpyAsync(&e, s->tc_err, sizeof e, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
      cudaStreamSynchronize(s->stream) != cudaSuccess)
    return sfail(s, MPM_ERR_CUDA, "reading the tensor-core kernels' status failed");
  if (e) {
    cudaMemsetAsync(s->tc_err, 0, sizeof(unsigned), s->stream);
    return sfail(s, MPM_ERR_TIMEOUT, "a tensor-core completion wait gave up (the network's work was not used)");
  }
  return MPM_OK;
}

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
  if (material->model != 4 && material->model != 5 && material->model != 10 && !mpm::learned_model(material->model))
    return MPM_ERR_UNSUPPORTED;
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
      cudaMalloc(&s->loss, 16) != cudaSuccess || cudaMalloc(&s->wbf, sizeof(surr::WeightsBf16)) != cudaSuccess ||
      cudaMalloc(&s->tc_err, sizeof(unsigned)) != cudaSuccess)
    return bail(MPM_ERR_OUT_OF_MEMORY);
  if (cudaMemset(s->tc_err, 0, sizeof(unsigned)) != cudaSuccess ||
      cudaFuncSetAttribute(surr::k_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(surr::TcSmem)) !=
          cudaSuccess)
    return bail(MPM_ERR_CUDA);
  if (cudaFuncSetAttribute(surr::k_gated, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(surr::GateSmem)) !=
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
  void* bufs[] = {s->params, s->grad, s->adam_m, s->adam_v, s->loss, s->wbf, s->tc_err};
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
  if (F && is_jc(s)) return sfail(s, MPM_ERR_UNSUPPORTED, "Johnson-Cook rows carry no trial F");
  const surr::SampleSpec sp = spec_of(cfg);
  float *dX = nullptr, *dY = nullptr, *dD = nullptr, *dep = nullptr, *dT = nullptr;
  SCUDA(s, cudaMalloc(&dX, n * 8 * sizeof(float)));
  SCUDA(s, cudaMalloc(&dY, n * 8 * sizeof(float)));
  if (F) {
    SCUDA(s, cudaMalloc(&dD, n * 9 * sizeof(float)));
    SCUDA(s, cudaMalloc(&dep, n * sizeof(float)));
    SCUDA(s, cudaMalloc(&dT, n * sizeof(float)));
  }
  if (is_jc(s))
    surr::k_samples_jc<<<s->num_sms * 8, 256, 0, s->stream>>>(s->mt, sp, n, dX, dY);
  else
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
  // J2 / thermal J2: the stress correction (6) and dep (weighted); Johnson-Cook: the root u alone
  const float w_j2[8] = {1, 1, 1, 1, 1, 1, (float)(cfg->dep_weight > 0 ? cfg->dep_weight : 1.0), 0};
  const float w_jc[8] = {1, 0, 0, 0, 0, 0, 0, 0};
  const float* w = is_jc(s) ? w_jc : w_j2;
  const surr::SampleSpec sp = spec_of(cfg);
  int rc = MPM_OK;
  cudaError_t e = cudaMemcpyAsync(wout, w, 8 * sizeof(float), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) {
    if (is_jc(s))
      surr::k_samples_jc<<<s->num_sms * 8, 256, 0, s->stream>>>(s->mt, sp, n, X, Y);
    else
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
    launch_train(s, X, Y, n, first, stride, cfg->batch, wout, dloss + t);
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
  return check_tc(s);
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
    launch_train(s, dX, dY, n, 0, 1, (int)n, dw, dl);
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
  return check_tc(s);
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
  if (is_jc(s))
    return sfail(s, MPM_ERR_UNSUPPORTED, "Johnson-Cook networks run inside the step (mpm_set_return_mode) or in "
                                         "mpm_surrogate_time: their return depends on the substep");
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
    const GateLaunch gl = gate_launch(s, use_mlp, n);
    surr::k_gated<<<gl.blocks, surr::kGateThreads, gl.smem, s->stream>>>(
        s->wbf, s->params, s->mt, s->sc, (float)gate_tol, use_mlp, n, dF, de, dT, dFo, ddep, dtau, dpath, dc, s->tc_err);
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
  return check_tc(s);
}

// Timing of the gated map against the exact map on n device-resident random trial states.
static int time_jc(mpm_surrogate* s, const mpm_surrogate_config* cfg, int64_t n, int32_t iters, double gate_tol,
                   double* ms_exact, double* ms_learned, mpm_gate_counts* counts) {
  const surr::SampleSpec sp = spec_of(cfg);
  const int newton = cfg->newton > 0 ? cfg->newton : 8;
  float* dep = nullptr;
  surr::GateOut* dc = nullptr;
  SCUDA(s, cudaMalloc(&dep, n * sizeof(float)));
  SCUDA(s, cudaMalloc(&dc, sizeof(surr::GateOut)));
  const int blocks = (int)std::min<long long>(s->num_sms * 8, (n + 255) / 256);
  cudaEvent_t ev[4];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaError_t e = cudaMemsetAsync(dc, 0, sizeof(surr::GateOut), s->stream);
  // the exact map: the reference's bisection for every plastic state; the learned map: the network
  // as warp-wide tensor-core tiles (the fused pass's code), the refinement, the gate and the
  // bisection for what it rejects. (A tcgen05 form with 128 states per tile measured 0.466 ms against
  // 0.417 ms on 4,096,000 states: the CTA-wide barriers around its MMA groups cost more than the
  // 10 kFLOP network saves.)
  auto launch = [&](int mode, surr::GateOut* cnt) {
    surr::k_gated_jc<<<blocks, 256, 0, s->stream>>>(s->wbf, s->params, s->mt, sp, (float)gate_tol, newton, mode, n, dep,
                                                    cnt);
  };
  for (int mode = 0; mode < 2 && e == cudaSuccess; ++mode) {
    for (int w = 0; w < 2; ++w) launch(mode, nullptr);
    cudaEventRecord(ev[2 * mode], s->stream);
    for (int it = 0; it < iters; ++it) launch(mode, (mode == 1 && it == 0) ? dc : nullptr);
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
  cudaFree(dep);
  cudaFree(dc);
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

int mpm_surrogate_time(mpm_surrogate* s, const mpm_surrogate_config* cfg, int64_t n, int32_t iters, double gate_tol,
                       double* ms_exact, double* ms_learned, mpm_gate_counts* counts) {
  if (!s || !cfg || n <= 0 || iters <= 0 || !ms_exact || !ms_learned) return MPM_ERR_INVALID_ARG;
  if (is_jc(s)) return time_jc(s, cfg, n, iters, gate_tol, ms_exact, ms_learned, counts);
  const surr::SampleSpec sp = spec_of(cfg);
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
  cudaEvent_t ev[4];
  for (auto& x : ev) cudaEventCreate(&x);
  for (int mode = 0; mode < 2 && e == cudaSuccess; ++mode) {
    for (int w = 0; w < 2; ++w)
      surr::k_gated<<<gate_launch(s, mode, n).blocks, surr::kGateThreads, gate_launch(s, mode, n).smem, s->stream>>>(
          s->wbf, s->params, s->mt, s->sc, (float)gate_tol, mode, n, dD, de, dT, dFo, ddep, dtau, nullptr, nullptr,
          s->tc_err);
    cudaMemsetAsync(dc, 0, sizeof(surr::GateOut), s->stream);
    cudaEventRecord(ev[2 * mode], s->stream);
    for (int it = 0; it < iters; ++it)
      surr::k_gated<<<gate_launch(s, mode, n).blocks, surr::kGateThreads, gate_launch(s, mode, n).smem, s->stream>>>(
          s->wbf, s->params, s->mt, s->sc, (float)gate_tol, mode, n, dD, de, dT, dFo, ddep, dtau, nullptr,
          it == 0 ? dc : nullptr, s->tc_err);
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
  return check_tc(s);
}

int mpm_surrogate_time_newton(mpm_surrogate* s, const mpm_surrogate_config* cfg, int64_t n, int32_t iters,
                              double gate_tol, double* ms, mpm_gate_counts* counts) {
  if (!s || !cfg || !ms || n <= 0 || iters <= 0 || !(gate_tol > 0)) return MPM_ERR_INVALID_ARG;
  if (!is_jc(s)) return sfail(s, MPM_ERR_UNSUPPORTED, "the Newton-gated map serves the Johnson-Cook laws (models 6, 7)");
  const surr::SampleSpec sp = spec_of(cfg);
  const int newton = cfg->newton > 0 ? cfg->newton : 8;
  float* dep = nullptr;
  surr::GateOut* dc = nullptr;
  SCUDA(s, cudaMalloc(&dep, n * sizeof(float)));
  SCUDA(s, cudaMalloc(&dc, sizeof(surr::GateOut)));
  const int blocks = (int)std::min<long long>(s->num_sms * 8, (n + 255) / 256);
  cudaEvent_t ev[2];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaError_t e = cudaMemsetAsync(dc, 0, sizeof(surr::GateOut), s->stream);
  for (int w = 0; w < 2 && e == cudaSuccess; ++w)
    surr::k_gated_jc<<<blocks, 256, 0, s->stream>>>(s->wbf, s->params, s->mt, sp, (float)gate_tol, newton, 2, n, dep,
                                                    nullptr);
  cudaEventRecord(ev[0], s->stream);
  for (int it = 0; it < iters && e == cudaSuccess; ++it)
    surr::k_gated_jc<<<blocks, 256, 0, s->stream>>>(s->wbf, s->params, s->mt, sp, (float)gate_tol, newton, 2, n, dep,
                                                    it == 0 ? dc : nullptr);
  cudaEventRecord(ev[1], s->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  surr::GateOut hc{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hc, dc, sizeof hc, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  float t = 0;
  if (e == cudaSuccess) cudaEventElapsedTime(&t, ev[0], ev[1]);
  for (auto& x : ev) cudaEventDestroy(x);
  cudaFree(dep);
  cudaFree(dc);
  if (e != cudaSuccess) return sfail(s, MPM_ERR_CUDA, cudaGetErrorString(e));
  *ms = t / iters;
  if (counts) {
    counts->elastic = hc.elastic;
    counts->learned = hc.learned;
    counts->fallback = hc.fallback;
  }
  return MPM_OK;
}

}  // extern "C"

namespace surr {

int surrogate_model(const mpm_surrogate* s) { return s ? s->mat.model : -1; }

size_t weights_bytes() { return sizeof(WeightsBf16); }

int export_weights(mpm_surrogate* s, void* dst_w, float* dst_params, cudaStream_t st) {
  if (!s || !dst_w || !dst_params) return MPM_ERR_INVALID_ARG;
  // the surrogate's own stream finishes its pending updates first
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return MPM_ERR_CUDA;
  if (cudaMemcpyAsync(dst_w, s->wbf, sizeof(WeightsBf16), cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(dst_params, s->params, kParams * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return MPM_ERR_CUDA;
  return MPM_OK;
}

}  // namespace surr
