// 2D elastic MLS-MPM solid: the drop-in for the reference's SolidMPM (src/solid-mpm.js:20-116).
//
// The reference steps at most 16,000 particles (src/simulation.js:7) on a fixed 149 x 149 node
// grid, so this path is bound by launch latency and host round trips, not by HBM. The design
// follows from that:
//   * F and C live on the device for the handle's lifetime (float4 each, one 16-byte load);
//     the caller's Float32 particle arrays cross PCIe once per call in each direction.
//   * The grid (m, px, py, fixed-mass) is a float4 per node, 355 KB, resident in L2; P2G adds
//     one float4 vector atomic per node per particle. The grid pass normalises, applies the
//     walls, writes node velocities and clears the accumulator in the same read, so no
//     separate clear launch exists.
//   * smpm_frame runs the whole MPM branch of Simulation.step on the device: G2P fuses the
//     next substep's stableStep reduction, and the last block to finish decides the next
//     substep length and whether the frame is done, so the host launches batches of substeps
//     and reads one small control block per batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "mpm_b200.h"

namespace {

constexpr int kN = 149;  // src/solid-mpm.js:4
constexpr int kNodes = kN * kN;
constexpr float kDX = 8.f, kOrigin = -592.f, kArea = 12.96f;
constexpr int kThreads = 128;
constexpr int kMaxSubsteps = 96;  // src/simulation.js:250
constexpr int kBatch = 4;         // substeps launched per host check

struct Ctrl2 {
  double remaining;  // frame time still to solve
  double h;          // length of the current substep
  int steps;         // substeps taken in this frame
  int done;
  int active_nodes;  // nodes with mass > 1e-12 in the last grid pass
  unsigned ticket;   // last-block-done counter
  unsigned wave_bits, grad_bits;  // stableStep maxima (non-negative floats compare as uints)
  // stats reduction
  unsigned count, minj_key, maxj_key, strain_bits;
};

struct Params2 {
  int count;
  int walls;
  float bound, floor_, top;
  int gravity;
  float force;  // 27 * settings.strength
  float sound;  // sqrt(19200 * solidStiffness)
  float stiffness;
  unsigned mask[8];  // MPM-solid material ids
};

struct Dev2 {
  float4 *F, *C;
  float *x, *y, *vx, *vy, *mass, *volume;
  uint8_t *material, *pinned;
  float4* grid;
  float2* vel;
  Ctrl2* ctrl;
};

__device__ __forceinline__ bool solid(const Params2& p, uint8_t m) { return (p.mask[m >> 5] >> (m & 31)) & 1u; }

__device__ __forceinline__ unsigned ordered_key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

struct St2 {
  int bx, by;
  float fx, fy, wx[3], wy[3];
};

// src/solid-mpm.js:30-36. The fraction is measured from the base node's position (an integer, so
// exact in FP32), not as (x - origin) / DX - base: x - origin is ~600 units, where one FP32 ulp is
// 6e-5 units, which would cost the fraction 7.6e-6 cells; x - node is exact or within one ulp of
// a number below 16.
__device__ __forceinline__ void stencil2(float x, float y, St2& s) {
  const float px = (x - kOrigin) * (1.f / kDX), py = (y - kOrigin) * (1.f / kDX);
  s.bx = min(max((int)floorf(px - .5f), 0), kN - 3);
  s.by = min(max((int)floorf(py - .5f), 0), kN - 3);
  s.fx = (x - (kOrigin + kDX * (float)s.bx)) * (1.f / kDX);
  s.fy = (y - (kOrigin + kDX * (float)s.by)) * (1.f / kDX);
  s.wx[0] = .5f * (1.5f - s.fx) * (1.5f - s.fx);
  s.wx[1] = .75f - (s.fx - 1.f) * (s.fx - 1.f);
  s.wx[2] = .5f * (s.fx - .5f) * (s.fx - .5f);
  s.wy[0] = .5f * (1.5f - s.fy) * (1.5f - s.fy);
  s.wy[1] = .75f - (s.fy - 1.f) * (s.fy - 1.f);
  s.wy[2] = .5f * (s.fy - .5f) * (s.fy - .5f);
}

// src/solid-mpm.js:10-18: Kirchhoff stress of 2D fixed-corotated elasticity, closed-form polar.
__host__ __device__ inline void solid_stress(float a, float b, float c, float d, float mu, float lambda, float* tau) {
  const float J = a * d - b * c, q = hypotf(a + d, c - b);
  const float r = q > 1e-12f ? (a + d) / q : 1.f, t = q > 1e-12f ? (c - b) / q : 0.f;
  const float volume = lambda * (J - 1.f) * J;
  tau[0] = 2.f * mu * ((a - r) * a + (b + t) * b) + volume;
  tau[1] = 2.f * mu * ((a - r) * c + (b + t) * d);
  tau[2] = 2.f * mu * ((c - t) * a + (d - r) * b);
  tau[3] = 2.f * mu * ((c - t) * c + (d - r) * d) + volume;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide max of two unsigned keys into global atomics.
__device__ void block_max2(unsigned a, unsigned b, unsigned* ga, unsigned* gb) {
  __shared__ unsigned sa[kThreads / 32], sb[kThreads / 32];
  a = warp_max(a);
  b = warp_max(b);
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = a;
    sb[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / 32; ++w) {
      a = max(a, sa[w]);
      b = max(b, sb[w]);
    }
    atomicMax(ga, a);
    atomicMax(gb, b);
  }
}

// stableStep terms of one particle (src/solid-mpm.js:40-44)
__device__ __forceinline__ void stable_terms(const Params2& p, float4 F, float4 C, float vx, float vy, unsigned& wave,
                                             unsigned& grad) {
  const float stretch = fmaxf(1.f, sqrtf(F.x * F.x + F.y * F.y + F.z * F.z + F.w * F.w));
  const float w = hypotf(vx, vy) + p.sound * stretch * stretch;
  const float g = fabsf(C.x) + fabsf(C.y) + fabsf(C.z) + fabsf(C.w);
  wave = max(wave, __float_as_uint(w));
  grad = max(grad, __float_as_uint(g));
}

// Last block of a stableStep reduction: the next substep length and the frame's done flag
// (src/solid-mpm.js:45, src/simulation.js:250-253). `advance` closes the substep that just ran.
__device__ void finish_stable(Ctrl2* c, bool advance) {
  __threadfence();
  if (atomicAdd(&c->ticket, 1u) != gridDim.x - 1) return;
  __threadfence();
  const float wave = fmaxf(1.f, __uint_as_float(atomicAdd(&c->wave_bits, 0u)));
  const float grad = __uint_as_float(atomicAdd(&c->grad_bits, 0u));
  if (advance) {
    c->remaining -= c->h;
    c->steps += 1;
  }
  const double stable = fmin(fmin(1.0 / 240, (double)(.18f * kDX / wave)), (double)(.1f / fmaxf(1.f, grad)));
  c->h = fmin(c->remaining, stable);
  c->done = !(c->remaining > 1e-9 && c->steps < kMaxSubsteps);
  c->wave_bits = 0;
  c->grad_bits = 0;
  c->ticket = 0;
}

// stableStep over the current state; with frame != 0 it also opens the frame's first substep.
__global__ void __launch_bounds__(kThreads) k2_stable(Dev2 d, Params2 p) {
  unsigned wave = 0, grad = 0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < p.count; i += gridDim.x * kThreads)
    if (solid(p, d.material[i])) stable_terms(p, d.F[i], d.C[i], d.vx[i], d.vy[i], wave, grad);
  block_max2(wave, grad, &d.ctrl->wave_bits, &d.ctrl->grad_bits);
  if (threadIdx.x == 0) finish_stable(d.ctrl, false);
}

// Body force of Simulation.substep for MPM solids (src/simulation.js:270-288, force != 0 only
// in frame mode) and the P2G scatter of src/solid-mpm.js:50-64.
__global__ void __launch_bounds__(kThreads) k2_p2g(Dev2 d, Params2 p, int frame) {
  const Ctrl2* c = d.ctrl;
  if (c->done) return;
  const float h = (float)c->h;
  if (blockIdx.x == 0 && threadIdx.x == 0) d.ctrl->active_nodes = 0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < p.count; i += gridDim.x * kThreads) {
    if (!solid(p, d.material[i])) continue;
    const bool pin = d.pinned[i] != 0;
    float x = d.x[i], y = d.y[i], vx = d.vx[i], vy = d.vy[i];
    if (frame) {
      if (pin) {
        vx = vy = 0.f;
      } else {
        float gx = 0.f, gy = 0.f;
        if (p.gravity == SMPM_GRAVITY_CENTER) {
          const float r = sqrtf(x * x + y * y + 400.f);
          gx = -x / r;
          gy = -y / r;
        } else if (p.gravity == SMPM_GRAVITY_UNIFORM) {
          gy = -1.f;
        }
        vx = fminf(fmaxf(vx + gx * p.force * h, -180.f), 180.f);
        vy = fminf(fmaxf(vy + gy * p.force * h, -180.f), 180.f);
      }
      d.vx[i] = vx;
      d.vy[i] = vy;
    }
    St2 s;
    stencil2(x, y, s);
    const float m = d.mass[i], V0 = kArea * d.volume[i], rho = m / V0, E = rho * 16000.f * p.stiffness;
    const float4 F = d.F[i], C = d.C[i];
    float tau[4];
    solid_stress(F.x, F.y, F.z, F.w, .4f * E, .4f * E, tau);
    const float factor = -h * V0 * 4.f / (kDX * kDX);
    const float a00 = m * C.x + factor * tau[0], a01 = m * C.y + factor * tau[1];
    const float a10 = m * C.z + factor * tau[2], a11 = m * C.w + factor * tau[3];
    const float pm = pin ? m : 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float w = s.wx[k] * s.wy[j], dx = ((float)k - s.fx) * kDX, dy = ((float)j - s.fy) * kDX;
        const int n = (s.by + j) * kN + s.bx + k;
        atomicAdd(&d.grid[n], make_float4(w * m, w * (m * vx + a00 * dx + a01 * dy), w * (m * vy + a10 * dx + a11 * dy),
                                          w * pm));
      }
  }
}

// Grid update of src/solid-mpm.js:65-76; clears the accumulator for the next P2G.
__global__ void __launch_bounds__(kThreads) k2_grid(Dev2 d, Params2 p) {
  if (d.ctrl->done) return;
  int active = 0;
  for (int n = blockIdx.x * kThreads + threadIdx.x; n < kNodes; n += gridDim.x * kThreads) {
    const float4 a = d.grid[n];
    d.grid[n] = make_float4(0.f, 0.f, 0.f, 0.f);
    float ux = a.y, uy = a.z;  // a node at or below the mass threshold keeps its raw sums
    if (a.x > 1e-12f) {
      ++active;
      ux /= a.x;
      uy /= a.x;
      if (a.w > 1e-9f) {
        ux = uy = 0.f;
      } else if (p.walls) {
        const float x = kOrigin + (float)(n % kN) * kDX, y = kOrigin + (float)(n / kN) * kDX;
        if ((x < -p.bound + kDX && ux < 0.f) || (x > p.bound - kDX && ux > 0.f)) ux = 0.f;
        if ((y < p.floor_ + kDX && uy < 0.f) || (y > p.top - kDX && uy > 0.f)) uy = 0.f;
      }
    }
    d.vel[n] = make_float2(ux, uy);
  }
  for (int o = 16; o; o >>= 1) active += __shfl_xor_sync(0xffffffffu, active, o);
  if ((threadIdx.x & 31) == 0 && active) atomicAdd(&d.ctrl->active_nodes, active);
}

// G2P with the C and F update (src/solid-mpm.js:77-90); in frame mode also the next stableStep.
__global__ void __launch_bounds__(kThreads) k2_g2p(Dev2 d, Params2 p, int frame) {
  if (d.ctrl->done) return;
  const float h = (float)d.ctrl->h;
  unsigned wave = 0, grad = 0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < p.count; i += gridDim.x * kThreads) {
    if (!solid(p, d.material[i])) continue;
    float4 F = d.F[i], C = d.C[i];
    float vx = d.vx[i], vy = d.vy[i];
    if (!d.pinned[i]) {
      float x = d.x[i], y = d.y[i];
      St2 s;
      stencil2(x, y, s);
      float gvx = 0.f, gvy = 0.f, a = 0.f, b = 0.f, c = 0.f, e = 0.f;
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const float2 u = d.vel[(s.by + j) * kN + s.bx + k];
          const float w = s.wx[k] * s.wy[j], dx = ((float)k - s.fx) * (4.f / kDX), dy = ((float)j - s.fy) * (4.f / kDX);
          gvx += w * u.x;
          gvy += w * u.y;
          a += w * u.x * dx;
          b += w * u.x * dy;
          c += w * u.y * dx;
          e += w * u.y * dy;
        }
      C = make_float4(a, b, c, e);
      F = make_float4((1.f + h * a) * F.x + h * b * F.z, (1.f + h * a) * F.y + h * b * F.w,
                      h * c * F.x + (1.f + h * e) * F.z, h * c * F.y + (1.f + h * e) * F.w);
      vx = gvx;
      vy = gvy;
      x += h * vx;
      y += h * vy;
      if (p.walls) {
        x = fminf(fmaxf(x, -p.bound + .1f), p.bound - .1f);
        y = fminf(fmaxf(y, p.floor_ + .1f), p.top - .1f);
      }
      d.F[i] = F;
      d.C[i] = C;
      d.vx[i] = vx;
      d.vy[i] = vy;
      d.x[i] = x;
      d.y[i] = y;
    }
    if (frame) stable_terms(p, F, C, vx, vy, wave, grad);
  }
  if (frame) {
    block_max2(wave, grad, &d.ctrl->wave_bits, &d.ctrl->grad_bits);
    if (threadIdx.x == 0) finish_stable(d.ctrl, true);
  }
}

// SolidMPM.stats reduction (src/solid-mpm.js:108-116)
__global__ void __launch_bounds__(kThreads) k2_stats(Dev2 d, Params2 p) {
  unsigned cnt = 0, mn = 0xffffffffu, mx = 0, st = 0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < p.count; i += gridDim.x * kThreads) {
    if (!solid(p, d.material[i])) continue;
    const float4 F = d.F[i];
    const float J = F.x * F.w - F.y * F.z;
    const float e0 = F.x * F.x + F.z * F.z - 1.f, e1 = F.y * F.y + F.w * F.w - 1.f,
                e2 = 1.41421356f * (F.x * F.y + F.z * F.w);
    ++cnt;
    mn = min(mn, ordered_key(J));
    mx = max(mx, ordered_key(J));
    st = max(st, __float_as_uint(.5f * sqrtf(e0 * e0 + e1 * e1 + e2 * e2)));
  }
  for (int o = 16; o; o >>= 1) {
    cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    st = max(st, __shfl_xor_sync(0xffffffffu, st, o));
  }
  if ((threadIdx.x & 31) == 0 && cnt) {
    atomicAdd(&d.ctrl->count, cnt);
    atomicMin(&d.ctrl->minj_key, mn);
    atomicMax(&d.ctrl->maxj_key, mx);
    atomicMax(&d.ctrl->strain_bits, st);
  }
}

__global__ void k2_reset(float4* F, float4* C, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    F[i] = make_float4(1.f, 0.f, 0.f, 1.f);
    C[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

}  // namespace

struct smpm_handle {
  long long capacity = 0;
  cudaStream_t stream = nullptr;
  Dev2 d{};
  Ctrl2* host_ctrl = nullptr;  // pinned
  unsigned mask[8] = {};
  int substeps = 0;  // SolidMPM.substeps: set by a frame
  int nodes = 0;     // SolidMPM.activeNodes: set by every grid pass
  std::string err;
  int fail(int rc, const std::string& what) {
    err = what;
    return rc;
  }
  int cuda(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return MPM_OK;
    err = std::string(where) + ": " + cudaGetErrorString(e);
    return MPM_ERR_CUDA;
  }
};

namespace {

int blocks_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + kThreads - 1) / kThreads, 1184)); }

int check_sim(smpm_handle* h, const smpm_sim* s) {
  if (!s) return h->fail(MPM_ERR_INVALID_ARG, "null sim");
  if (s->count < 0 || s->count > h->capacity) return h->fail(MPM_ERR_CAPACITY, "count exceeds the handle's capacity");
  if (s->count > 0 && (!s->x || !s->y || !s->vx || !s->vy || !s->mass || !s->volume || !s->material || !s->pinned))
    return h->fail(MPM_ERR_INVALID_ARG, "null particle array");
  if (!(s->solid_stiffness >= 0) || !std::isfinite(s->solid_stiffness))
    return h->fail(MPM_ERR_INVALID_ARG, "solid_stiffness must be finite and >= 0");
  return MPM_OK;
}

Params2 params_of(const smpm_handle* h, const smpm_sim* s) {
  Params2 p{};
  p.count = s->count;
  const bool demo = s->scene == SMPM_SCENE_SOFTBODY, basin = s->scene == SMPM_SCENE_BASIN;
  p.walls = (s->boundary || demo || basin) ? 1 : 0;
  p.bound = demo ? 170.f : basin ? 245.f : 555.f;  // src/solid-mpm.js:66
  p.floor_ = demo ? -145.f : basin ? -175.f : -555.f;
  p.top = demo ? 145.f : p.bound;
  p.gravity = s->gravity;
  p.force = (float)(27.0 * s->strength);
  p.sound = (float)std::sqrt(19200.0 * s->solid_stiffness);
  p.stiffness = (float)s->solid_stiffness;
  std::memcpy(p.mask, h->mask, sizeof p.mask);
  return p;
}

int upload_sim(smpm_handle* h, const smpm_sim* s) {
  const size_t n = (size_t)s->count;
  if (!n) return MPM_OK;
  cudaStream_t st = h->stream;
  const size_t f = n * sizeof(float);
  cudaError_t e = cudaSuccess;
  e = e ? e : cudaMemcpyAsync(h->d.x, s->x, f, cudaMemcpyHostToDevice, st);
  e = e ? e : cudaMemcpyAsync(h->d.y, s->y, f, cudaMemcpyHostToDevice, st);
  e = e ? e : cudaMemcpyAsync(h->d.vx, s->vx, f, cudaMemcpyHostToDevice, st);
  e = e ? e : cudaMemcpyAsync(h->d.vy, s->vy, f, cudaMemcpyHostToDevice, st);
  e = e ? e : cudaMemcpyAsync(h->d.mass, s->mass, f, cudaMemcpyHostToDevice, st);
  e = e ? e : cudaMemcpyAsync(h->d.volume, s->volume, f, cudaMemcpyHostToDevice, st);
  e = e ? e : cudaMemcpyAsync(h->d.material, s->material, n, cudaMemcpyHostToDevice, st);
  e = e ? e : cudaMemcpyAsync(h->d.pinned, s->pinned, n, cudaMemcpyHostToDevice, st);
  return h->cuda(e, "copy particles in");
}

int download_sim(smpm_handle* h, const smpm_sim* s) {
  const size_t f = (size_t)s->count * sizeof(float);
  cudaStream_t st = h->stream;
  cudaError_t e = cudaSuccess;
  if (f) {
    e = e ? e : cudaMemcpyAsync(s->x, h->d.x, f, cudaMemcpyDeviceToHost, st);
    e = e ? e : cudaMemcpyAsync(s->y, h->d.y, f, cudaMemcpyDeviceToHost, st);
    e = e ? e : cudaMemcpyAsync(s->vx, h->d.vx, f, cudaMemcpyDeviceToHost, st);
    e = e ? e : cudaMemcpyAsync(s->vy, h->d.vy, f, cudaMemcpyDeviceToHost, st);
  }
  e = e ? e : cudaMemcpyAsync(h->host_ctrl, h->d.ctrl, sizeof(Ctrl2), cudaMemcpyDeviceToHost, st);
  e = e ? e : cudaStreamSynchronize(st);
  if (e == cudaSuccess) h->nodes = h->host_ctrl->active_nodes;
  return h->cuda(e, "copy particles out");
}

int set_ctrl(smpm_handle* h, double remaining, double step) {
  Ctrl2 c{};
  c.remaining = remaining;
  c.h = step;
  c.minj_key = 0xffffffffu;
  *h->host_ctrl = c;
  cudaError_t e = cudaMemcpyAsync(h->d.ctrl, h->host_ctrl, sizeof(Ctrl2), cudaMemcpyHostToDevice, h->stream);
  // the pinned block is rewritten by the next read-back only after this copy completes
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return h->cuda(e, "control block");
}

}  // namespace

extern "C" {

int smpm_create(int64_t capacity, smpm_handle** out) {
  if (!out || capacity <= 0 || capacity > (1ll << 31) - 1) return MPM_ERR_INVALID_ARG;
  *out = nullptr;
  smpm_handle* h = new smpm_handle();
  h->capacity = capacity;
  h->mask[11 >> 5] |= 1u << (11 & 31);  // MATERIALS[11].mpm (src/materials.js:15)
  const size_t n = (size_t)capacity;
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  e = e ? e : cudaMalloc(&h->d.F, n * sizeof(float4));
  e = e ? e : cudaMalloc(&h->d.C, n * sizeof(float4));
  float** fl[6] = {&h->d.x, &h->d.y, &h->d.vx, &h->d.vy, &h->d.mass, &h->d.volume};
  for (float** a : fl) e = e ? e : cudaMalloc(a, n * sizeof(float));
  e = e ? e : cudaMalloc(&h->d.material, n);
  e = e ? e : cudaMalloc(&h->d.pinned, n);
  e = e ? e : cudaMalloc(&h->d.grid, kNodes * sizeof(float4));
  e = e ? e : cudaMalloc(&h->d.vel, kNodes * sizeof(float2));
  e = e ? e : cudaMalloc(&h->d.ctrl, sizeof(Ctrl2));
  e = e ? e : cudaMallocHost(&h->host_ctrl, sizeof(Ctrl2));
  e = e ? e : cudaMemsetAsync(h->d.grid, 0, kNodes * sizeof(float4), h->stream);
  e = e ? e : cudaMemsetAsync(h->d.ctrl, 0, sizeof(Ctrl2), h->stream);
  if (e == cudaSuccess) {
    k2_reset<<<blocks_for(capacity), kThreads, 0, h->stream>>>(h->d.F, h->d.C, capacity);
    e = cudaGetLastError();
  }
  e = e ? e : cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    smpm_destroy(h);
    return e == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA;
  }
  *out = h;
  return MPM_OK;
}

int smpm_destroy(smpm_handle* h) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (h->stream) cudaStreamSynchronize(h->stream);
  void* bufs[] = {h->d.F, h->d.C, h->d.x, h->d.y, h->d.vx, h->d.vy, h->d.mass, h->d.volume,
                  h->d.material, h->d.pinned, h->d.grid, h->d.vel, h->d.ctrl};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (h->host_ctrl) cudaFreeHost(h->host_ctrl);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return MPM_OK;
}

const char* smpm_last_error(const smpm_handle* h) { return h ? h->err.c_str() : "null handle"; }

int smpm_set_mpm_materials(smpm_handle* h, const uint8_t* ids, int32_t n) {
  if (!h || n < 0 || (n > 0 && !ids)) return MPM_ERR_INVALID_ARG;
  std::memset(h->mask, 0, sizeof h->mask);
  for (int i = 0; i < n; ++i) h->mask[ids[i] >> 5] |= 1u << (ids[i] & 31);
  return MPM_OK;
}

int smpm_reset(smpm_handle* h) {
  if (!h) return MPM_ERR_INVALID_ARG;
  k2_reset<<<blocks_for(h->capacity), kThreads, 0, h->stream>>>(h->d.F, h->d.C, h->capacity);
  cudaError_t e = cudaGetLastError();
  e = e ? e : cudaMemsetAsync(h->d.ctrl, 0, sizeof(Ctrl2), h->stream);
  e = e ? e : cudaStreamSynchronize(h->stream);
  h->substeps = h->nodes = 0;
  return h->cuda(e, "reset");
}

int smpm_reset_particle(smpm_handle* h, int64_t i) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (i < 0 || i >= h->capacity) return h->fail(MPM_ERR_OUT_OF_RANGE, "particle index out of range");
  static const float4 I = {1.f, 0.f, 0.f, 1.f}, Z = {0.f, 0.f, 0.f, 0.f};
  cudaError_t e = cudaMemcpyAsync(h->d.F + i, &I, sizeof(float4), cudaMemcpyHostToDevice, h->stream);
  e = e ? e : cudaMemcpyAsync(h->d.C + i, &Z, sizeof(float4), cudaMemcpyHostToDevice, h->stream);
  e = e ? e : cudaStreamSynchronize(h->stream);
  return h->cuda(e, "reset particle");
}

int smpm_remove_particle(smpm_handle* h, int64_t i, int64_t last) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (i < 0 || i >= h->capacity || last < 0 || last >= h->capacity)
    return h->fail(MPM_ERR_OUT_OF_RANGE, "particle index out of range");
  cudaError_t e = cudaMemcpyAsync(h->d.F + i, h->d.F + last, sizeof(float4), cudaMemcpyDeviceToDevice, h->stream);
  e = e ? e : cudaMemcpyAsync(h->d.C + i, h->d.C + last, sizeof(float4), cudaMemcpyDeviceToDevice, h->stream);
  e = e ? e : cudaStreamSynchronize(h->stream);
  return h->cuda(e, "remove particle");
}

int smpm_has_particles(smpm_handle* h, const smpm_sim* s, int32_t* out) {
  if (!h || !out) return MPM_ERR_INVALID_ARG;
  int rc = check_sim(h, s);
  if (rc) return rc;
  *out = 0;
  for (int i = 0; i < s->count; ++i)
    if ((h->mask[s->material[i] >> 5] >> (s->material[i] & 31)) & 1u) {
      *out = 1;
      break;
    }
  return MPM_OK;
}

int smpm_stable_step(smpm_handle* h, const smpm_sim* s, double* dt) {
  if (!h || !dt) return MPM_ERR_INVALID_ARG;
  int rc = check_sim(h, s);
  if (rc || (rc = upload_sim(h, s)) || (rc = set_ctrl(h, INFINITY, 0.0))) return rc;
  const Params2 p = params_of(h, s);
  k2_stable<<<blocks_for(s->count), kThreads, 0, h->stream>>>(h->d, p);
  cudaError_t e = cudaGetLastError();
  e = e ? e : cudaMemcpyAsync(h->host_ctrl, h->d.ctrl, sizeof(Ctrl2), cudaMemcpyDeviceToHost, h->stream);
  e = e ? e : cudaStreamSynchronize(h->stream);
  if ((rc = h->cuda(e, "stable step"))) return rc;
  *dt = h->host_ctrl->h;
  return MPM_OK;
}

int smpm_step(smpm_handle* h, const smpm_sim* s, double dt) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!std::isfinite(dt) || dt < 0) return h->fail(MPM_ERR_INVALID_ARG, "dt must be finite and >= 0");
  int rc = check_sim(h, s);
  if (rc || (rc = upload_sim(h, s)) || (rc = set_ctrl(h, dt, dt))) return rc;
  const Params2 p = params_of(h, s);
  k2_p2g<<<blocks_for(s->count), kThreads, 0, h->stream>>>(h->d, p, 0);
  k2_grid<<<blocks_for(kNodes), kThreads, 0, h->stream>>>(h->d, p);
  k2_g2p<<<blocks_for(s->count), kThreads, 0, h->stream>>>(h->d, p, 0);
  if ((rc = h->cuda(cudaGetLastError(), "step launch"))) return rc;
  return download_sim(h, s);
}

int smpm_frame(smpm_handle* h, const smpm_sim* s, double dt, int32_t* substeps, double* advanced) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!std::isfinite(dt)) return h->fail(MPM_ERR_INVALID_ARG, "dt must be finite");
  if (s && s->gravity != SMPM_GRAVITY_NONE && s->gravity != SMPM_GRAVITY_CENTER && s->gravity != SMPM_GRAVITY_UNIFORM)
    return h->fail(MPM_ERR_UNSUPPORTED, "gravity mode not supported by the MPM frame");
  int rc = check_sim(h, s);
  dt = std::min(std::max(dt, 0.0), 0.05);  // src/simulation.js:241
  if (rc || (rc = upload_sim(h, s)) || (rc = set_ctrl(h, dt, 0.0))) return rc;
  const Params2 p = params_of(h, s);
  const int pb = blocks_for(s->count), gb = blocks_for(kNodes);
  k2_stable<<<pb, kThreads, 0, h->stream>>>(h->d, p);
  for (int launched = 0; launched < kMaxSubsteps;) {
    for (int k = 0; k < kBatch && launched < kMaxSubsteps; ++k, ++launched) {
      k2_p2g<<<pb, kThreads, 0, h->stream>>>(h->d, p, 1);
      k2_grid<<<gb, kThreads, 0, h->stream>>>(h->d, p);
      k2_g2p<<<pb, kThreads, 0, h->stream>>>(h->d, p, 1);
    }
    cudaError_t e = cudaGetLastError();
    e = e ? e : cudaMemcpyAsync(h->host_ctrl, h->d.ctrl, sizeof(Ctrl2), cudaMemcpyDeviceToHost, h->stream);
    e = e ? e : cudaStreamSynchronize(h->stream);
    if ((rc = h->cuda(e, "frame"))) return rc;
    if (h->host_ctrl->done) break;
  }
  if ((rc = download_sim(h, s))) return rc;
  h->substeps = h->host_ctrl->steps;
  if (substeps) *substeps = h->host_ctrl->steps;
  if (advanced) *advanced = dt - h->host_ctrl->remaining;
  return MPM_OK;
}

int smpm_stats_get(smpm_handle* h, const smpm_sim* s, smpm_stats* out) {
  if (!h || !out) return MPM_ERR_INVALID_ARG;
  int rc = check_sim(h, s);
  if (rc) return rc;
  if (s->count > 0) {
    cudaError_t e = cudaMemcpyAsync(h->d.material, s->material, (size_t)s->count, cudaMemcpyHostToDevice, h->stream);
    if ((rc = h->cuda(e, "stats input"))) return rc;
  }
  if ((rc = set_ctrl(h, 0.0, 0.0))) return rc;
  const Params2 p = params_of(h, s);
  k2_stats<<<blocks_for(s->count), kThreads, 0, h->stream>>>(h->d, p);
  cudaError_t e = cudaGetLastError();
  e = e ? e : cudaMemcpyAsync(h->host_ctrl, h->d.ctrl, sizeof(Ctrl2), cudaMemcpyDeviceToHost, h->stream);
  e = e ? e : cudaStreamSynchronize(h->stream);
  if ((rc = h->cuda(e, "stats"))) return rc;
  const Ctrl2& r = *h->host_ctrl;
  auto key_to_float = [](unsigned k) {
    const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  };
  out->count = (int32_t)r.count;
  out->min_j = r.count ? key_to_float(r.minj_key) : 1.0;
  out->max_j = r.count ? key_to_float(r.maxj_key) : 1.0;
  float strain;
  std::memcpy(&strain, &r.strain_bits, 4);
  out->strain = strain;
  out->nodes = h->nodes;
  out->substeps = h->substeps;
  out->pad = 0;
  return MPM_OK;
}

int smpm_get_fields(smpm_handle* h, int64_t n, double* fields) {
  if (!h || n < 0 || (n > 0 && !fields)) return MPM_ERR_INVALID_ARG;
  if (n > h->capacity) return h->fail(MPM_ERR_CAPACITY, "n exceeds the handle's capacity");
  std::vector<float4> F(n), C(n);
  cudaError_t e = cudaSuccess;
  if (n) {
    e = cudaMemcpyAsync(F.data(), h->d.F, n * sizeof(float4), cudaMemcpyDeviceToHost, h->stream);
    e = e ? e : cudaMemcpyAsync(C.data(), h->d.C, n * sizeof(float4), cudaMemcpyDeviceToHost, h->stream);
  }
  e = e ? e : cudaStreamSynchronize(h->stream);
  int rc = h->cuda(e, "get fields");
  if (rc) return rc;
  for (int64_t i = 0; i < n; ++i) {
    const float v[8] = {F[i].x, F[i].y, F[i].z, F[i].w, C[i].x, C[i].y, C[i].z, C[i].w};
    for (int k = 0; k < 8; ++k) fields[k * n + i] = v[k];
  }
  return MPM_OK;
}

int smpm_set_fields(smpm_handle* h, int64_t n, const double* fields) {
  if (!h || n < 0 || (n > 0 && !fields)) return MPM_ERR_INVALID_ARG;
  if (n > h->capacity) return h->fail(MPM_ERR_CAPACITY, "n exceeds the handle's capacity");
  std::vector<float4> F(n), C(n);
  for (int64_t i = 0; i < n; ++i) {
    F[i] = make_float4((float)fields[i], (float)fields[n + i], (float)fields[2 * n + i], (float)fields[3 * n + i]);
    C[i] = make_float4((float)fields[4 * n + i], (float)fields[5 * n + i], (float)fields[6 * n + i], (float)fields[7 * n + i]);
  }
  cudaError_t e = cudaSuccess;
  if (n) {
    e = cudaMemcpyAsync(h->d.F, F.data(), n * sizeof(float4), cudaMemcpyHostToDevice, h->stream);
    e = e ? e : cudaMemcpyAsync(h->d.C, C.data(), n * sizeof(float4), cudaMemcpyHostToDevice, h->stream);
  }
  e = e ? e : cudaStreamSynchronize(h->stream);  // the host vectors die at return
  return h->cuda(e, "set fields");
}

}  // extern "C"
