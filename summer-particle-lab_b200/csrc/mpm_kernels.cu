// CUDA kernels of the B200-native MLS-MPM solid step (sm_100a).
//
// One substep is five launches on one stream (all persistent or grid-stride, no host sync):
//   k_begin        1 CTA: dt from the device-side CFL maxima, step bookkeeping, list resets
//   k_grid_update  active node tiles only: v = (p + dt (f + m g)) / m, walls, sticky floor
//   k_g2p2g        per particle tile: TMA-staged 6^3 velocity window -> gather v, C -> F update
//                  -> advect -> constitutive update / J2 return -> scatter m, p, f of the new
//                  state into an 8^3 shared-memory window -> one float4 atomic per node per tile;
//                  emits the next sort key and the next CFL maxima
//   k_scan         exclusive scan of per-tile counts (last-block-done, one launch)
//   k_sort_scatter counting sort: perm[start + rank] = particle, first claimer appends the tile
//                  to the work list
// The scatter is dt-free (m, p = sum w (m v + m C dpos), f = -sum w (4V/h) tau dpos), so the next
// substep's dt can be chosen on the device after the whole state is known, as the reference does
// (src/three/simulation.js:308-310); the grid update applies dt.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "mpm_internal.h"
#include "surrogate_net.h"

namespace mpm {

// ---------------------------------------------------------------------------------------------
// small device helpers

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `limit` SM cycles (default 2^31, about 1 s) and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  long long limit = 1ll << 31) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

// Self-check of the bounded wait: one thread waits on an mbarrier that nothing arrives on, gives
// up after `limit` cycles and reports 1 in out[0] (0 would mean the wait completed).
__global__ void k_wait_probe(unsigned* out, long long limit) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  fence_barrier_init();
  out[0] = mbar_wait_bounded(&bar, 0, limit) ? 0u : 1u;
}

void launch_wait_probe(cudaStream_t st, unsigned* out, long long limit) { k_wait_probe<<<1, 32, 0, st>>>(out, limit); }

// 4D tiled TMA load (no multicast): box {4 channels, 6, 6, 6} of the grid velocity array.
// The innermost coordinate is the channel index 0, so the 16-byte alignment rule holds.
__device__ __forceinline__ void tma_load_4d(void* dst, const void* tmap, int c0, int c1, int c2, int c3,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
      "%4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ int find_scene_by_tile(const SceneDev* sc, int ns, int t) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sc[mid].tile_base <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int find_scene_by_node_tile(const SceneDev* sc, int ns, int t) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sc[mid].node_tile_base <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Paired FP32 arithmetic of sm_100 (FFMA2 / FMUL2): two independent lanes per instruction, each
// rounded exactly like a scalar fmaf / multiply, so the results are bitwise those of the scalar form.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 dup2(float x) { return make_float2(x, x); }

// Stencil along one axis from a fixed-point position (src/three/mpm.js:25-32):
// base = clamp(floor(q - 0.5), 0, N - 3), t = q - base (exact: integer below 2^24 times 2^-22).
__device__ __forceinline__ void stencil_axis(unsigned q, int dim, int& base, float& t) {
  int b = (q < (1u << (kFracBits - 1))) ? -1 : static_cast<int>((q - (1u << (kFracBits - 1))) >> kFracBits);
  b = min(max(b, 0), dim - 3);
  base = b;
  t = static_cast<float>(static_cast<long long>(q) - (static_cast<long long>(b) << kFracBits)) * kInvFixedOne;
}

__device__ __forceinline__ unsigned tile_key(const SceneDev& sc, const int b[3]) {
  return static_cast<unsigned>(sc.tile_base) +
         static_cast<unsigned>(((b[2] >> 2) * sc.tiles[1] + (b[1] >> 2)) * sc.tiles[0] + (b[0] >> 2));
}

__device__ __forceinline__ void mark_node_tile(const Ctx& c, unsigned tile, int list) {
  if (atomicExch(&c.g.tile_flag[tile], 1u) == 0u) {
    const unsigned idx = atomicAdd(&c.ctrl->active_count[list], 1u);
    c.g.active[list][idx] = tile;
  }
}

__device__ __forceinline__ void mark_node_tiles_of(const Ctx& c, const SceneDev& sc, int n0, int n1, int n2,
                                                   int list) {
  // node tiles covering nodes [n, n+2] on each axis
  for (int tz = n2 >> 2; tz <= (n2 + 2) >> 2; ++tz)
    for (int ty = n1 >> 2; ty <= (n1 + 2) >> 2; ++ty)
      for (int tx = n0 >> 2; tx <= (n0 + 2) >> 2; ++tx)
        mark_node_tile(c, sc.node_tile_base + (tz * sc.ntiles[1] + ty) * sc.ntiles[0] + tx, list);
}

// Warp-aggregated increment of the per-tile particle count.
__device__ __forceinline__ void count_key(const Ctx& c, unsigned key) {
  const unsigned mask = __match_any_sync(0xffffffffu, key);
  const int lane = threadIdx.x & 31;
  if (key != 0xffffffffu && lane == __ffs(mask) - 1) atomicAdd(&c.s.count[key], __popc(mask));
}

__device__ __forceinline__ double warp_sum_d(double x) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__device__ __forceinline__ unsigned fbits(float x) { return __float_as_uint(fmaxf(x, 0.f)); }

// CFL terms of src/three/mpm.js:43-54 for one particle (F = I + D)
template <bool AUX>
__device__ __forceinline__ void cfl_terms(const MaterialDev& mt, const float D[9], const float v[3],
                                          const float C[9], float m, float V, float Jm1, float aux, float& wave,
                                          float& grad) {
  float row = 0.f, col = 0.f, g = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float r = 0.f, cc = 0.f;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      r += fabsf(D[a * 3 + b] + (a == b ? 1.f : 0.f));
      cc += fabsf(D[b * 3 + a] + (a == b ? 1.f : 0.f));
      g += fabsf(C[a * 3 + b]);
    }
    row = fmaxf(row, r);
    col = fmaxf(col, cc);
  }
  // Neo-Hookean and the pressure models stiffen in compression (by J, or J Jp for 8 and 9); snow's
  // moduli carry its hardening
  const bool press = AUX && (mt.model == 8 || mt.model == 9);
  const float compression = mt.model == 1 || press ? 1.f / fmaxf(0.05f, (1.f + Jm1) * (press ? 1.f + aux : 1.f)) : 1.f;
  const float c = sqrtf(mt.wave_modulus * (AUX && mt.model == 2 ? snow_hardening(aux) : 1.f) * V / m);
  const float speed = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  wave = speed + c * fmaxf(1.f, fmaxf(row * col, compression));
  grad = g;
}

// ---------------------------------------------------------------------------------------------
// control

struct ControlOp {
  int op;           // 0: reset lists for an initial sort + P2G, 1: start a step call
  int mode;
  double dt_requested;
  int max_substeps;  // per requested-dt step in requested mode, per call otherwise
  float dt_fixed;
  int nsteps;        // requested-dt steps in this call
};

__global__ void k_control(Ctx c, ControlOp op) {
  Ctrl* ct = c.ctrl;
  if (threadIdx.x == 0) {
    const unsigned k = ct->step_index;
    ct->last_substep = 1u;
    if (op.op == 0) {
      ct->work_count[k & 1] = 0;
      ct->active_count[k & 1] = 0;
      ct->work_next = 0;
      ct->done = 0;
    } else {
      ct->remaining = op.dt_requested;
      ct->dt_requested = op.dt_requested;
      ct->advanced = 0.0;
      ct->substeps = 0;
      ct->max_substeps = op.max_substeps;
      ct->done = 0;
      ct->mode = op.mode;
      ct->dt_fixed = op.dt_fixed;
      ct->steps_left = op.nsteps > 1 ? op.nsteps : 1;
      ct->step_substeps = 0;
    }
  }
  if (op.op == 0) {
    for (int s = threadIdx.x; s < c.nscenes; s += blockDim.x) {
      c.wave_max[s] = 0u;
      c.grad_max[s] = 0u;
    }
  }
}

void launch_control_init(const Ctx& c, cudaStream_t st) {
  ControlOp op{0, 0, 0.0, 0, 0.f, 1};
  k_control<<<1, 256, 0, st>>>(c, op);
}

void launch_control_step(const Ctx& c, cudaStream_t st, int mode, double dt_req, int max_substeps, float dt_fixed,
                         int nsteps) {
  ControlOp op{1, mode, dt_req, max_substeps, dt_fixed, nsteps};
  k_control<<<1, 32, 0, st>>>(c, op);
}

// Substep prologue: picks dt per scene, or marks the call done.
__global__ void __launch_bounds__(256) k_begin(Ctx c) {
  Ctrl* ct = c.ctrl;
  __shared__ float smin[8];
  __shared__ int sdone;
  __shared__ float sdt;
  if (ct->done) return;
  if (ct->status & 0x8u) {  // a bounded wait gave up: stop this call
    if (threadIdx.x == 0) ct->done = 1;
    return;
  }
  float local = 3.0e38f;
  for (int s = threadIdx.x; s < c.nscenes; s += blockDim.x) {
    const SceneDev& sc = c.scenes[s];
    const float wave = fmaxf(1.f, __uint_as_float(c.wave_max[s]));
    const float grad = fmaxf(1.f, __uint_as_float(c.grad_max[s]));
    float dt = fminf(sc.dt_max, fminf(sc.cfl * sc.H / wave, sc.grad_limit / grad));
    if (sc.cond_G > 0.f) dt = fminf(dt, sc.cond_dt_max);
    c.dt_scene[s] = dt;  // provisional: the scene's own stable dt
    local = fminf(local, dt);
  }
  for (int o = 16; o > 0; o >>= 1) local = fminf(local, __shfl_xor_sync(0xffffffffu, local, o));
  if ((threadIdx.x & 31) == 0) smin[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x == 0) {
    float m = smin[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fminf(m, smin[w]);
    int done = 0;
    float dt = m;
    if (ct->mode == kModeRequested) {
      // a requested-dt step ends when its time is used up or it has taken max_substeps; the
      // call's next step (mpm_run) then starts with the full requested dt
      bool over = !(ct->remaining > 1e-6 * ct->dt_requested) || ct->step_substeps >= ct->max_substeps;
      if (over && ct->steps_left > 1) {
        ct->steps_left -= 1;
        ct->remaining = ct->dt_requested;
        ct->step_substeps = 0;
        over = false;
      }
      if (over) done = 1;
      dt = static_cast<float>(fmin(ct->remaining, static_cast<double>(m)));
      if (!done) {
        // the last substep takes exactly what is left (src/three/simulation.js:309)
        if (ct->remaining - dt <= 1e-6 * ct->dt_requested) dt = static_cast<float>(ct->remaining);
        ct->remaining -= dt;
      }
    } else {
      if (ct->substeps >= ct->max_substeps) done = 1;
      if (ct->mode == kModeFixed) dt = ct->dt_fixed;
    }
    if (done) {
      ct->done = 1;
    } else {
      ct->substeps += 1;
      ct->step_substeps += 1;
      ct->advanced += dt;
      // the next k_begin ends the call after this substep (the same tests it will make)
      bool last;
      if (ct->mode == kModeRequested)
        last = ct->steps_left <= 1 &&
               (!(ct->remaining > 1e-6 * ct->dt_requested) || ct->step_substeps >= ct->max_substeps);
      else
        last = ct->substeps >= ct->max_substeps;
      ct->last_substep = last ? 1u : 0u;
      const unsigned k = ct->step_index + 1;
      ct->step_index = k;
      ct->work_count[k & 1] = 0;
      ct->active_count[k & 1] = 0;
      ct->work_next = 0;
      ct->grid_next = 0;
    }
    sdone = done;
    sdt = dt;
  }
  __syncthreads();
  if (sdone) return;
  for (int s = threadIdx.x; s < c.nscenes; s += blockDim.x) {
    if (ct->mode != kModeCfl || c.uniform_dt) c.dt_scene[s] = sdt;
    c.time_scene[s] += static_cast<double>(c.dt_scene[s]);
    c.wave_max[s] = 0u;
    c.grad_max[s] = 0u;
  }
}

void launch_begin(const Ctx& c, cudaStream_t st) { k_begin<<<1, 256, 0, st>>>(c); }

// ---------------------------------------------------------------------------------------------
// counting sort by particle tile

__global__ void __launch_bounds__(256) k_keys(Ctx c) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned key = 0xffffffffu;
  if (i < c.n) {
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, i);
    const SceneDev& sc = c.scenes[s];
    int b[3];
    float t;
    stencil_axis(c.p.qx[i], sc.dims[0], b[0], t);
    stencil_axis(c.p.qy[i], sc.dims[1], b[1], t);
    stencil_axis(c.p.qz[i], sc.dims[2], b[2], t);
    key = tile_key(sc, b);
    c.p.key[i] = key;
  }
  count_key(c, key);
}

void launch_keys(const Ctx& c, cudaStream_t st) {
  const long long blocks = (c.n + 255) / 256;
  if (blocks > 0) k_keys<<<static_cast<unsigned>(blocks), 256, 0, st>>>(c);
}

constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int kScanChunk = kScanThreads * kScanPer;  // 4096 tiles per block

// Exclusive scans of count[0..T] into start (block-local) + block_off (per 4096 tiles), and of the
// non-empty flags into rank + block_rank (a tile's place in the work list, which so comes out in
// tile-key order). The last block to finish scans the block sums (threadfence + ticket) and sets
// the work list's length.
// initial: the scan of a first sort (done is clear); otherwise the scan after a scatter pass, which
// may run beside the next substep's opening kernels and so reads the pass's own flag, not done.
__device__ __forceinline__ uint2 warp_incl_scan2(uint2 v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned a = __shfl_up_sync(0xffffffffu, v.x, o);
    const unsigned b = __shfl_up_sync(0xffffffffu, v.y, o);
    if (lane >= o) {
      v.x += a;
      v.y += b;
    }
  }
  return v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan(Ctx c, int initial) {
  if (initial ? c.ctrl->done != 0 : c.ctrl->sort_active == 0) return;
  if (c.ctrl->status & 0x8u) return;
  __shared__ uint2 warp_sums[32];
  __shared__ bool last;
  const int T = c.total_tiles + 1;
  const int base = blockIdx.x * kScanChunk + threadIdx.x * kScanPer;
  unsigned v[kScanPer];
  uint2 sum = make_uint2(0u, 0u);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    v[k] = (base + k < c.total_tiles) ? c.s.count[base + k] : 0u;
    sum.x += v[k];
    sum.y += v[k] > 0u ? 1u : 0u;
  }
  // block exclusive scan of per-thread sums
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint2 incl = warp_incl_scan2(sum, lane);
  if (lane == 31) warp_sums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const uint2 ws = warp_sums[lane];
    const uint2 wi = warp_incl_scan2(ws, lane);
    warp_sums[lane] = make_uint2(wi.x - ws.x, wi.y - ws.y);
  }
  __syncthreads();
  uint2 run = make_uint2(warp_sums[wid].x + incl.x - sum.x, warp_sums[wid].y + incl.y - sum.y);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < T) {
      c.s.start[base + k] = run.x;
      c.s.rank[base + k] = run.y;
    }
    run.x += v[k];
    run.y += v[k] > 0u ? 1u : 0u;
  }
  if (threadIdx.x == kScanThreads - 1) {  // block totals
    c.s.block_off[blockIdx.x] = run.x;
    c.s.block_rank[blockIdx.x] = run.y;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(&c.ctrl->scan_ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  // last block: exclusive scan of the block totals (gridDim.x <= 1024 * 64 blocks)
  __shared__ uint2 carry;
  if (threadIdx.x == 0) carry = make_uint2(0u, 0u);
  __syncthreads();
  for (int b0 = 0; b0 < (int)gridDim.x; b0 += kScanThreads) {
    const int b = b0 + threadIdx.x;
    const uint2 x = (b < (int)gridDim.x)
                        ? make_uint2(*((volatile unsigned*)&c.s.block_off[b]), *((volatile unsigned*)&c.s.block_rank[b]))
                        : make_uint2(0u, 0u);
    const uint2 inc = warp_incl_scan2(x, lane);
    if (lane == 31) warp_sums[wid] = inc;
    __syncthreads();
    if (wid == 0) {
      const uint2 ws = warp_sums[lane];
      const uint2 wi = warp_incl_scan2(ws, lane);
      warp_sums[lane] = make_uint2(wi.x - ws.x, wi.y - ws.y);
    }
    __syncthreads();
    const uint2 excl = make_uint2(carry.x + warp_sums[wid].x + inc.x - x.x, carry.y + warp_sums[wid].y + inc.y - x.y);
    if (b < (int)gridDim.x) {
      c.s.block_off[b] = excl.x;
      c.s.block_rank[b] = excl.y;
    }
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry = make_uint2(excl.x + x.x, excl.y + x.y);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const unsigned list = initial ? (c.ctrl->step_index & 1u) : c.ctrl->sort_list;
    c.ctrl->work_count[list] = carry.y;  // non-empty tiles
    c.ctrl->scan_ticket = 0;
  }
}

void launch_scan(const Ctx& c, cudaStream_t st, bool initial) {
  const int blocks = (c.total_tiles + 1 + kScanChunk - 1) / kScanChunk;
  k_scan<<<blocks, kScanThreads, 0, st>>>(c, initial ? 1 : 0);
}

__device__ __forceinline__ unsigned tile_start(const Ctx& c, unsigned k) {
  return c.s.start[k] + c.s.block_off[k / kScanChunk];
}

// perm[start(k) + rank] = home slot; the group that claims a tile first writes its work item.
// After a scatter pass the sort may run beside the next substep's k_begin and grid update, so it
// takes its list and its go-ahead from the fields that pass wrote (sort_list, sort_active), which
// k_begin does not touch.
__global__ void __launch_bounds__(256) k_sort_scatter(Ctx c, int initial) {
  if (!initial && c.ctrl->sort_active == 0) return;
  if (c.ctrl->status & 0x8u) return;  // a bounded wait gave up this substep
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const unsigned key = i < c.n ? c.p.key[i] : 0xffffffffu;
  const unsigned mask = __match_any_sync(0xffffffffu, key);
  if (key == 0xffffffffu) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  const unsigned below = __popc(mask & ((1u << lane) - 1u));
  const unsigned group = __popc(mask);
  unsigned old = 0;
  if (lane == leader) old = atomicSub(&c.s.count[key], group);
  old = __shfl_sync(mask, old, leader);
  const unsigned s0 = tile_start(c, key);
  const unsigned cnt = tile_start(c, key + 1) - s0;
  // counts and keys always agree; a mismatch is reported and the write skipped
  if (old < below + 1 || old > cnt || static_cast<long long>(s0) + old - 1 - below >= c.n) {
    atomicOr(&c.ctrl->status, 0x20u);
    return;
  }
  c.p.perm[s0 + old - 1 - below] = static_cast<unsigned>(i);
  if (lane == leader && old == cnt) {  // the tile's first group writes its work item at the tile's rank
    const unsigned list = initial ? (c.ctrl->step_index & 1u) : c.ctrl->sort_list;
    const unsigned idx = c.s.rank[key] + c.s.block_rank[key / kScanChunk];
    const int s = c.nscenes == 1 ? 0 : find_scene_by_tile(c.scenes, c.nscenes, static_cast<int>(key));
    if (idx < static_cast<unsigned>(c.total_tiles)) c.s.work[list][idx] = make_uint4(key, s0, cnt, static_cast<unsigned>(s));
  }
}

void launch_sort_scatter(const Ctx& c, cudaStream_t st, bool initial) {
  const long long blocks = (c.n + 255) / 256;
  if (blocks > 0) k_sort_scatter<<<static_cast<unsigned>(blocks), 256, 0, st>>>(c, initial ? 1 : 0);
}

// ---------------------------------------------------------------------------------------------
// particle kernels
//
// One persistent kernel template serves the three particle passes:
//   kPassP2G    scatter of the current state (stress from F without a return)
//   kPassG2P2G  gather -> F update -> advect -> return map -> scatter of the new state
//   kPassG2P    gather -> F update -> advect -> return map (no scatter; host round-trip steps)
// Scatter in two phases per tile (up to kCap particles per round):
//   A  thread per particle: compute the new state and a 22-float payload (fraction t, m, m v,
//      m C h, -4V/h tau); bucket it by its stencil base inside the 8^3 scatter window
//      (shared-memory counting sort, native integer atomics)
//   B  thread per (non-empty base bucket, z layer): all particles of a bucket hit the same 27
//      nodes, so the 9 nodes x 7 channels of one layer are summed in registers and written with
//      63 shared atomics per bucket and layer (about 24 per particle instead of 189)
// then one float4 atomic per touched node and channel group flushes the window to HBM.

// Particles per scatter round. A full tile holds 512 (64 cells x 8), but a block that drifts by a
// fraction of a cell leaves a third of its tiles a few particles over 512 (up to ~530); at
// kCap = 512 those took a second round (every phase and barrier again for a handful of particles).
constexpr int kCap = 768;
constexpr int kPf = 2;         // perm entries of the next tile's first round held per thread (shared memory)
// Payload of one particle: 12 float pairs, laid out for the paired FMAs of phase B:
//   0 (tx, ty)   1 (tz, m)    2 (mv0, mv1)  3 (mv2, m T)  [m T only with conduction, else 0]
//   4 (c02, c12) 5 (c22, s02) 6 (s12, s22)  7 (c01, c11)  8 (c21, s01)  9 (c00, c10)  10 (c20, s00)
//   11 (s11, 0)
// with c = m h C and s = -4 V / h tau (symmetric).
constexpr int kPayRows = 12;
constexpr int kBuckets = 216;  // 6^3 possible stencil bases in the scatter window
// Payload slot of particle j: one extra word every 32 slots, so the slots phase B reads at a
// stride of a bucket's size (8 for the particles of one cell in consecutive slots) fall in
// different shared-memory banks; phase A's consecutive slots stay conflict-free.
constexpr int kPayStride = kCap + kCap / 32;
__device__ __forceinline__ int pay_slot(int j) { return j + (j >> 5); }
constexpr unsigned kMetaInvalid = 0x80000000u;

enum Pass : int { kPassP2G = 0, kPassG2P2G = 1, kPassG2P = 2 };

// Per-tile constants copied out of the scene table (kept in shared memory for the whole tile).
struct TileCtx {
  int tile[3];
  int dims[3];
  int gdim[3];
  unsigned qlo[3], qhi[3];
  long long node_base;
  float H, invH;
  int clamp;
  int mat;  // material row of a single-material scene
};

struct __align__(128) PartSmem {
  float4 vwin[2][kWinG * kWinG * kWinG];  // double-buffered TMA destinations (3456 B each)
  float acc[kChannels * kWinSNodes];      // 16 KiB scatter window
  float2 pay[kPayRows * kPayStride];      // 74 KiB payloads, structure of pair arrays (swizzled slots)
  unsigned meta[kCap];                    // bucket | rank << 8 (or kMetaInvalid)
  unsigned short sidx[kCap];              // slots sorted by bucket
  int hist[kBuckets];
  int bstart[kBuckets + 1];
  unsigned short blist[kBuckets];
  int nbuckets;
  int wsum[kBlock / 32], wnz[kBlock / 32];  // per-warp bucket totals of the block-wide scan
  unsigned long long mbar[2];
  uint4 item[2];
  int abort_flag;
  unsigned red[3 * (kBlock / 32)];
  unsigned gate[2];  // learned mode: returns the gate accepted / sent to the bisection
  // State the CTA carries from tile to tile sits here rather than in registers: at 128 registers a
  // thread, every register held across the tiles is one fewer for phase A, and moving these (with
  // the heat sum, which was a per-thread double) cut the pass by 7%.
  unsigned tma_phase[2];       // mbarrier phases of the two window buffers (thread 0)
  double work_sum;             // heat from plastic work of the CTA's particles
  int mt_row;                  // material row held in mt
  int pf_ok;                   // pfs holds the next tile's first-round perm entries
  unsigned pfs[kPf * kBlock];  // perm entries j of the next tile's first round, j < kPf x kBlock

  TileCtx tc;
  MaterialDev mt;
};

size_t particle_smem_bytes() { return sizeof(PartSmem); }
static_assert(sizeof(PartSmem) <= 112 * 1024, "two CTAs per SM");

// Direct global scatter (rare: particles that left the window, pinned particles): 27 nodes x
// channel atomics straight to the accumulators, and the node tiles they touch become active.
__device__ __noinline__ void scatter_global(const Ctx& c, const SceneDev& sc, const TileCtx& tc, int nxt,
                                               const int b[3], const float t[3], float m, const float mv[3],
                                               const float mC[9], const float s6[6], bool pinned, float mT) {
  float w[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) bspline_weights(t[a], w[a]);
  for (int kz = 0; kz < 3; ++kz)
    for (int ky = 0; ky < 3; ++ky)
      for (int kx = 0; kx < 3; ++kx) {
        const float dx = kx - t[0], dy = ky - t[1], dz = kz - t[2];
        const float wt = w[0][kx] * w[1][ky] * w[2][kz];
        const long long node = tc.node_base + ((long long)(b[2] + kz) * tc.gdim[1] + (b[1] + ky)) * tc.gdim[0] + (b[0] + kx);
        float* a0 = reinterpret_cast<float*>(&c.g.acc0[nxt][node]);
        float* a1 = reinterpret_cast<float*>(&c.g.acc1[nxt][node]);
        atomicAdd(a0 + 0, wt * m);
        atomicAdd(a0 + 1, wt * (mv[0] + mC[0] * dx + mC[1] * dy + mC[2] * dz));
        atomicAdd(a0 + 2, wt * (mv[1] + mC[3] * dx + mC[4] * dy + mC[5] * dz));
        atomicAdd(a0 + 3, wt * (mv[2] + mC[6] * dx + mC[7] * dy + mC[8] * dz));
        atomicAdd(a1 + 0, wt * (s6[0] * dx + s6[3] * dy + s6[4] * dz));
        atomicAdd(a1 + 1, wt * (s6[3] * dx + s6[1] * dy + s6[5] * dz));
        atomicAdd(a1 + 2, wt * (s6[4] * dx + s6[5] * dy + s6[2] * dz));
        if (pinned && wt > 1e-8f) atomicAdd(a1 + 3, wt * m);
        if (c.conduct) atomicAdd(&c.g.heat[nxt][node], wt * mT);
      }
  mark_node_tiles_of(c, sc, b[0], b[1], b[2], nxt);
}

// Flush the shared scatter window of one tile to the global accumulators (one float4 atomic per
// touched node and channel group) and clear it; mark the 27 node tiles it covers as active.
// tid / nthreads: this thread's index among the threads that flush.
__device__ __forceinline__ void flush_window_p(const Ctx& c, const SceneDev& sc, float* acc, int nxt, const int tile[3],
                                               int tid, int nthreads) {
  const int o0 = tile[0] * kTile - 1, o1 = tile[1] * kTile - 1, o2 = tile[2] * kTile - 1;
  for (int i = tid; i < kWinSNodes; i += nthreads) {
    const float mass = acc[i];
    if (mass != 0.f) {
      const int x = o0 + (i & 7), y = o1 + ((i >> 3) & 7), z = o2 + (i >> 6);
      if (x >= 0 && y >= 0 && z >= 0) {
        const long long node = sc.node_base + ((long long)z * sc.gdim[1] + y) * sc.gdim[0] + x;
        atomicAdd(&c.g.acc0[nxt][node], make_float4(mass, acc[1 * kWinSNodes + i], acc[2 * kWinSNodes + i],
                                                    acc[3 * kWinSNodes + i]));
        // channel 7 of the window is pinned mass without conduction (always zero there: pinned particles
        // scatter globally) and the heat sum w m T with it
        const float ch7 = acc[7 * kWinSNodes + i];
        atomicAdd(&c.g.acc1[nxt][node], make_float4(acc[4 * kWinSNodes + i], acc[5 * kWinSNodes + i],
                                                    acc[6 * kWinSNodes + i], c.conduct ? 0.f : ch7));
        if (c.conduct) atomicAdd(&c.g.heat[nxt][node], ch7);
      }
    }
#pragma unroll
    for (int ch = 0; ch < kChannels; ++ch) acc[ch * kWinSNodes + i] = 0.f;
  }
  if (tid < 27) {
    const int dx = tid % 3 - 1, dy = (tid / 3) % 3 - 1, dz = tid / 9 - 1;
    const int tx = tile[0] + dx, ty = tile[1] + dy, tz = tile[2] + dz;
    if (tx >= 0 && ty >= 0 && tz >= 0 && tx < sc.ntiles[0] && ty < sc.ntiles[1] && tz < sc.ntiles[2])
      mark_node_tile(c, sc.node_tile_base + (tz * sc.ntiles[1] + ty) * sc.ntiles[0] + tx, nxt);
  }
}

__device__ __forceinline__ void flush_window(const Ctx& c, const SceneDev& sc, PartSmem& sm, int nxt,
                                             const int tile[3]) {
  flush_window_p(c, sc, sm.acc, nxt, tile, threadIdx.x, kBlock);
}

// Block reduction of the per-thread CFL maxima and status flags of one tile, then one atomic per
// tile and scene. Every thread of the CTA calls it.
__device__ __forceinline__ void block_reduce_item(const Ctx& c, int scene, float wave, float grad, unsigned flags,
                                                  unsigned* red) {
  const unsigned wb = __reduce_max_sync(0xffffffffu, fbits(wave));
  const unsigned gb = __reduce_max_sync(0xffffffffu, fbits(grad));
  const unsigned fl = __reduce_or_sync(0xffffffffu, flags);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[wid * 3 + 0] = wb;
    red[wid * 3 + 1] = gb;
    red[wid * 3 + 2] = fl;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned w = 0, g = 0, f = 0;
    for (int k = 0; k < kBlock / 32; ++k) {
      w = max(w, red[k * 3 + 0]);
      g = max(g, red[k * 3 + 1]);
      f |= red[k * 3 + 2];
    }
    atomicMax(&c.wave_max[scene], w);
    atomicMax(&c.grad_max[scene], g);
    if (f) atomicOr(&c.ctrl->status, f);
  }
}

__device__ __forceinline__ unsigned state_flags(const float v[3], const float D[9], const Sym3& tau, float Jm1) {
  float s = v[0] + v[1] + v[2] + tau.xx + tau.yy + tau.zz + tau.xy + tau.xz + tau.yz;
#pragma unroll
  for (int k = 0; k < 9; ++k) s += D[k];
  unsigned f = 0;
  if (!isfinite(s)) f |= 0x1u;
  if (!(Jm1 > -1.f)) f |= 0x2u;
  return f;
}

// Phase B task: one non-empty base bucket, one z layer of its stencil. Sums the 3x3 nodes x 7
// channels over the bucket's particles in registers, then adds them to the shared window. The
// channels run as one scalar (mass) and three pairs (p0, p1), (p2, f0), (f1, f2) of paired FMAs.
template <bool HEAT>
__device__ __forceinline__ void bucket_layer_p(const float2* pay, const unsigned short* sidx, const int* bstart,
                                               float* acc, int b, int kz) {
  const int lx = b % 6, ly = (b / 6) % 6, lz = b / 36;
  float a0[3][3];
  float2 a12[3][3], a34[3][3], a56[3][3];
#pragma unroll
  for (int y = 0; y < 3; ++y)
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      a0[y][x] = 0.f;
      a12[y][x] = a34[y][x] = a56[y][x] = dup2(0.f);
    }
  const int i1 = bstart[b + 1];
  for (int i = bstart[b]; i < i1; ++i) {
    const int j = sidx[i];
    const float2* P = pay + pay_slot(j);
    const float2 txy = P[0 * kPayStride], tzm = P[1 * kPayStride], mv01 = P[2 * kPayStride];
    const float2 mv2h = P[3 * kPayStride], E = P[4 * kPayStride], Fz = P[5 * kPayStride];
    const float2 G = P[6 * kPayStride], H = P[7 * kPayStride], I = P[8 * kPayStride];
    const float2 K = P[9 * kPayStride], L = P[10 * kPayStride], S11 = P[11 * kPayStride];
    const float2 J = make_float2(S11.x, G.x);  // (s11, s12)
    const float2 M = make_float2(I.y, Fz.y);   // (s01, s02)
    float wx[3], wy[3], wzv[3];
    bspline_weights(txy.x, wx);
    bspline_weights(txy.y, wy);
    bspline_weights(tzm.x, wzv);
    const float wz = kz == 0 ? wzv[0] : (kz == 1 ? wzv[1] : wzv[2]);
    const float2 dz2 = dup2(static_cast<float>(kz) - tzm.x);
    const float2 q01 = ffma2(E, dz2, mv01);                        // (mv0 + c02 dz, mv1 + c12 dz)
    const float2 q2g0 = ffma2(Fz, dz2, make_float2(mv2h.x, 0.f));  // (mv2 + c22 dz, s02 dz)
    const float2 g12 = fmul2(G, dz2);                              // (s12 dz, s22 dz)
    const float mwz = tzm.y * wz;
#pragma unroll
    for (int y = 0; y < 3; ++y) {
      const float2 dy2 = dup2(static_cast<float>(y) - txy.y);
      const float wyz = wy[y] * wz;
      const float2 p01 = ffma2(H, dy2, q01), p2f0 = ffma2(I, dy2, q2g0), f12 = ffma2(J, dy2, g12);
      const float mwyz = mwz * wy[y];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        const float2 dx2 = dup2(static_cast<float>(x) - txy.x);
        const float2 wt = dup2(wx[x] * wyz);
        a0[y][x] = fmaf(wx[x], mwyz, a0[y][x]);
        a12[y][x] = ffma2(wt, ffma2(K, dx2, p01), a12[y][x]);
        a34[y][x] = ffma2(wt, ffma2(L, dx2, p2f0), a34[y][x]);
        a56[y][x] = ffma2(wt, ffma2(M, dx2, f12), a56[y][x]);
      }
    }
  }
#pragma unroll
  for (int y = 0; y < 3; ++y)
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      float* A = acc + ((lz + kz) * kWinS + (ly + y)) * kWinS + (lx + x);
      atomicAdd(A + 0 * kWinSNodes, a0[y][x]);
      atomicAdd(A + 1 * kWinSNodes, a12[y][x].x);
      atomicAdd(A + 2 * kWinSNodes, a12[y][x].y);
      atomicAdd(A + 3 * kWinSNodes, a34[y][x].x);
      atomicAdd(A + 4 * kWinSNodes, a34[y][x].y);
      atomicAdd(A + 5 * kWinSNodes, a56[y][x].x);
      atomicAdd(A + 6 * kWinSNodes, a56[y][x].y);
    }
  if (HEAT) {  // sum w m T into channel 7 (conduction)
    float hsum[3][3];
#pragma unroll
    for (int y = 0; y < 3; ++y)
#pragma unroll
      for (int x = 0; x < 3; ++x) hsum[y][x] = 0.f;
    for (int i = bstart[b]; i < i1; ++i) {
      const float2* P = pay + pay_slot(sidx[i]);
      const float2 txy = P[0 * kPayStride];
      float wx[3], wy[3], wzv[3];
      bspline_weights(txy.x, wx);
      bspline_weights(txy.y, wy);
      bspline_weights(P[1 * kPayStride].x, wzv);
      const float wmt = (kz == 0 ? wzv[0] : (kz == 1 ? wzv[1] : wzv[2])) * P[3 * kPayStride].y;
#pragma unroll
      for (int y = 0; y < 3; ++y)
#pragma unroll
        for (int x = 0; x < 3; ++x) hsum[y][x] += wx[x] * wy[y] * wmt;
    }
#pragma unroll
    for (int y = 0; y < 3; ++y)
#pragma unroll
      for (int x = 0; x < 3; ++x)
        atomicAdd(&acc[7 * kWinSNodes + ((lz + kz) * kWinS + (ly + y)) * kWinS + (lx + x)], hsum[y][x]);
  }
}

template <bool HEAT>
__device__ __forceinline__ void bucket_layer(PartSmem& sm, int b, int kz) {
  bucket_layer_p<HEAT>(sm.pay, sm.sidx, sm.bstart, sm.acc, b, kz);
}

// Exclusive scan of the bucket histogram over a group of NT >= kBuckets threads, with the compact
// list of non-empty buckets: thread t takes bucket t, warps scan their 32 buckets, and each thread
// adds the totals of the warps before it (one group barrier, `sync`). A one-warp scan here left the
// other warps of the group idle for a quarter of the pass. With clear, the histogram is zeroed for
// the next round on the way (it is not read after the scan).
template <int NT, typename Sync>
__device__ __forceinline__ void scan_buckets_group(int* hist, int* bstart, unsigned short* blist, int* nbuckets,
                                                   int* wsum, int* wnz, int t, bool clear, Sync&& sync) {
  static_assert(NT >= kBuckets && NT % 32 == 0, "one thread per bucket");
  const int lane = t & 31, w = t >> 5;
  const int h = t < kBuckets ? hist[t] : 0;
  if (clear && t < kBuckets) hist[t] = 0;
  int inc = h;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  const unsigned nz = __ballot_sync(0xffffffffu, h > 0);
  if (lane == 31) {
    wsum[w] = inc;
    wnz[w] = __popc(nz);
  }
  sync();
  int base = 0, nbase = 0;
  for (int k = 0; k < w; ++k) {
    base += wsum[k];
    nbase += wnz[k];
  }
  if (t < kBuckets) bstart[t] = base + inc - h;
  if (h > 0) blist[nbase + __popc(nz & ((1u << lane) - 1u))] = static_cast<unsigned short>(t);
  if (t == NT - 1) {
    bstart[kBuckets] = base + inc;
    *nbuckets = nbase + __popc(nz);
  }
}

__device__ __forceinline__ void scan_buckets(PartSmem& sm) {
  scan_buckets_group<kBlock>(sm.hist, sm.bstart, sm.blist, &sm.nbuckets, sm.wsum, sm.wnz, threadIdx.x, true,
                             [] { __syncthreads(); });
}


// Weighted gather of the 27 stencil nodes: out = (v, C / (4/h)) with v = sum w v_i and
// C_ab = sum w v_i,a (i - t)_b (src/three/mpm.js:110-117). The tensor-product weights are contracted
// one axis at a time (x, then y, then z), which needs about 280 FMAs instead of 430.
// ld(kz, ky, kx) returns the node velocity.
template <typename Ld>
__device__ __forceinline__ void gather27(Ld ld, const float t[3], const float w[3][3], float out[12]) {
  const float dx[3] = {-t[0], 1.f - t[0], 2.f - t[0]};
  const float dy[3] = {-t[1], 1.f - t[1], 2.f - t[1]};
  const float dz[3] = {-t[2], 1.f - t[2], 2.f - t[2]};
  const float wxd[3] = {w[0][0] * dx[0], w[0][1] * dx[1], w[0][2] * dx[2]};
  float v0 = 0.f, v1 = 0.f, v2 = 0.f;
  float cx0 = 0.f, cx1 = 0.f, cx2 = 0.f, cy0 = 0.f, cy1 = 0.f, cy2 = 0.f, cz0 = 0.f, cz1 = 0.f, cz2 = 0.f;
#pragma unroll
  for (int kz = 0; kz < 3; ++kz) {
    float s00 = 0.f, s01 = 0.f, s02 = 0.f;  // sum_y wy r0
    float s10 = 0.f, s11 = 0.f, s12 = 0.f;  // sum_y wy r1
    float s20 = 0.f, s21 = 0.f, s22 = 0.f;  // sum_y wy dy r0
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
      float r00 = 0.f, r01 = 0.f, r02 = 0.f, r10 = 0.f, r11 = 0.f, r12 = 0.f;
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) {
        const float4 g = ld(kz, ky, kx);
        r00 = fmaf(w[0][kx], g.x, r00); r01 = fmaf(w[0][kx], g.y, r01); r02 = fmaf(w[0][kx], g.z, r02);
        r10 = fmaf(wxd[kx], g.x, r10); r11 = fmaf(wxd[kx], g.y, r11); r12 = fmaf(wxd[kx], g.z, r12);
      }
      const float wy = w[1][ky], wyd = wy * dy[ky];
      s00 = fmaf(wy, r00, s00); s01 = fmaf(wy, r01, s01); s02 = fmaf(wy, r02, s02);
      s10 = fmaf(wy, r10, s10); s11 = fmaf(wy, r11, s11); s12 = fmaf(wy, r12, s12);
      s20 = fmaf(wyd, r00, s20); s21 = fmaf(wyd, r01, s21); s22 = fmaf(wyd, r02, s22);
    }
    const float wz = w[2][kz], wzd = wz * dz[kz];
    v0 = fmaf(wz, s00, v0); v1 = fmaf(wz, s01, v1); v2 = fmaf(wz, s02, v2);
    cx0 = fmaf(wz, s10, cx0); cx1 = fmaf(wz, s11, cx1); cx2 = fmaf(wz, s12, cx2);
    cy0 = fmaf(wz, s20, cy0); cy1 = fmaf(wz, s21, cy1); cy2 = fmaf(wz, s22, cy2);
    cz0 = fmaf(wzd, s00, cz0); cz1 = fmaf(wzd, s01, cz1); cz2 = fmaf(wzd, s02, cz2);
  }
  // out[3 + 3a + b] = C_ab (velocity component a, offset axis b)
  out[0] = v0; out[1] = v1; out[2] = v2;
  out[3] = cx0; out[4] = cy0; out[5] = cz0;
  out[6] = cx1; out[7] = cy1; out[8] = cz1;
  out[9] = cx2; out[10] = cy2; out[11] = cz2;
}

// Weighted sum of the nodes' fourth channel (the conduction temperature increment).
template <typename Ld>
__device__ __forceinline__ float gather_w27(Ld ld, const float w[3][3]) {
  float sz = 0.f;
#pragma unroll
  for (int kz = 0; kz < 3; ++kz) {
    float sy = 0.f;
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
      float sx = 0.f;
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) sx = fmaf(w[0][kx], ld(kz, ky, kx).w, sx);
      sy = fmaf(w[1][ky], sx, sy);
    }
    sz = fmaf(w[2][kz], sy, sz);
  }
  return sz;
}

// Gather straight from global memory (a particle whose stencil is outside the staged window). The
// fractions come by value and the result returns by value, so the caller's arrays keep no address.
struct Gather12 {
  float v[12];
};
__device__ __noinline__ Gather12 gather_global(const float4* base, int sy, long long sz, float t0, float t1, float t2) {
  const float t[3] = {t0, t1, t2};
  float w[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) bspline_weights(t[a], w[a]);
  Gather12 g;
  gather27([&](int kz, int ky, int kx) { return base[kz * sz + ky * sy + kx]; }, t, w, g.v);
  return g;
}

// Phase A of one particle (home slot `home`, payload row j): G2P from the staged window, F update,
// fixed-point advection and the constitutive update / return map (src/three/mpm.js:107-131), or,
// for the P2G pass and pinned particles, the stress of the stored state; then the scatter payload
// bucketed by its new stencil base in the shared window (pay, meta, hist), and the CFL terms.
// Writes the particle's new state and returns its next sort key (all ones when not needed).
// NEWTON (the Newton-gated return mode): a Johnson-Cook trial stress above the initial flow stress
// takes the gated refinement from u0 = 1 - flow(ep, 0, T) / q instead of the bisection, which stays
// the fallback; gate[0] / gate[1] count the returns accepted / sent to the bisection.
template <int PASS, bool HEAT, bool AUX, bool NEWTON = false>
__device__ __forceinline__ unsigned particle_phase_a(const Ctx& c, const SceneDev& sc, const TileCtx& tc,
                                                     const MaterialDev& mt_single, bool single, const float4* vwin,
                                                     unsigned home, unsigned j, float dt, int nxt, float2* pay,
                                                     unsigned* meta, int* hist, float& wave_acc, float& grad_acc,
                                                     unsigned& flags_acc, double& work_acc, bool store_vc,
                                                     unsigned* gate = nullptr) {
  static_assert(!NEWTON || (!HEAT && !AUX && PASS != kPassP2G), "Newton-gated returns: J2-type laws, gather passes");
  constexpr bool SCATTER = PASS != kPassG2P;
  constexpr bool GATHER = PASS != kPassP2G;
  unsigned key = 0xffffffffu;
  unsigned q[3] = {c.p.qx[home], c.p.qy[home], c.p.qz[home]};
  float D[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) D[e] = c.p.Dc[e][home];
  const float m = c.p.m[home], V = c.p.V[home];
  const MaterialDev& mt = single ? mt_single : c.mats[c.p.mat[home]];
  const MaterialExt* xp = AUX ? &c.mats_ext[single ? tc.mat : c.p.mat[home]] : nullptr;
  const bool pinned = c.has_pinned && c.p.pinned[home];
  float ep = c.has_plastic ? c.p.ep[home] : 0.f;
  float T = c.has_thermal ? c.p.T[home] : 0.f;
  float aux = AUX ? c.p.aux[home] : 0.f;
  float v[3], C[9];
  ConstitutiveOut co;
  unsigned flags = 0;
  if (GATHER && !pinned) {
    int b[3];
    float t[3], w[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      stencil_axis(q[a], tc.dims[a], b[a], t[a]);
      bspline_weights(t[a], w[a]);
    }
    const int l0 = b[0] - tc.tile[0] * kTile, l1 = b[1] - tc.tile[1] * kTile, l2 = b[2] - tc.tile[2] * kTile;
    // the sort key places the stencil inside the staged window; if it ever does not, the
    // particle reads the grid from global memory instead (and the step reports it)
    const bool in_g = l0 >= 0 && l0 <= kWinG - 3 && l1 >= 0 && l1 <= kWinG - 3 && l2 >= 0 && l2 <= kWinG - 3;
    if (!in_g) flags |= 0x20u;
    // G2P (src/three/mpm.js:107-118): v = sum w v_i, C = sum w v_i (i - t)^T 4/h
    float acc12[12];
    if (in_g) {
      const float4* win = &vwin[(l2 * kWinG + l1) * kWinG + l0];
      gather27([&](int kz, int ky, int kx) { return win[(kz * kWinG + ky) * kWinG + kx]; }, t, w, acc12);
    } else {
      const Gather12 g = gather_global(c.g.vel + tc.node_base + ((long long)b[2] * tc.gdim[1] + b[1]) * tc.gdim[0] + b[0],
                                       tc.gdim[0], (long long)tc.gdim[0] * tc.gdim[1], t[0], t[1], t[2]);
#pragma unroll
      for (int e = 0; e < 12; ++e) acc12[e] = g.v[e];
    }
    // grid heat conduction: the node temperature increments, interpolated like the velocity, and
    // relaxation of the particle's offset from the interpolated node temperature at the rate of the
    // finest unresolved mode (wavelength 2h): beta = 1 - exp(-pi^2 alpha dt / h^2); both parts keep
    // the heat sum, and the relaxation lets a body reach a uniform temperature
    if (HEAT && sc.cond_G > 0.f) {
      const long long o = tc.node_base + ((long long)b[2] * tc.gdim[1] + b[1]) * tc.gdim[0] + b[0];
      const long long sz = (long long)tc.gdim[0] * tc.gdim[1];
      float dTc;
      if (in_g) {
        const float4* win = &vwin[(l2 * kWinG + l1) * kWinG + l0];
        dTc = gather_w27([&](int kz, int ky, int kx) { return win[(kz * kWinG + ky) * kWinG + kx]; }, w);
      } else {
        const float4* base = c.g.vel + o;
        dTc = gather_w27([&](int kz, int ky, int kx) { return base[kz * sz + ky * tc.gdim[0] + kx]; }, w);
      }
      const float* tn = c.g.tnode + o;
      const float Tint = gather_w27([&](int kz, int ky, int kx) {
        return make_float4(0.f, 0.f, 0.f, tn[kz * sz + ky * tc.gdim[0] + kx]); }, w);
      const float beta = 1.f - expf(-9.8696044f * sc.cond_G * sc.cond_inv_mfull * sc.cond_inv_cp * dt);
      T += dTc + beta * (Tint - T);
    }
    const float v0 = acc12[0], v1 = acc12[1], v2 = acc12[2];
    const float c0 = acc12[3], c1 = acc12[4], c2 = acc12[5], c3 = acc12[6], c4 = acc12[7], c5 = acc12[8],
                c6 = acc12[9], c7 = acc12[10], c8 = acc12[11];
    const float s4 = 4.f * tc.invH;
    v[0] = v0; v[1] = v1; v[2] = v2;
    C[0] = c0 * s4; C[1] = c1 * s4; C[2] = c2 * s4;
    C[3] = c3 * s4; C[4] = c4 * s4; C[5] = c5 * s4;
    C[6] = c6 * s4; C[7] = c7 * s4; C[8] = c8 * s4;
    // F <- (I + dt C) F in centred form: D <- D + dt C (I + D) (src/three/mpm.js:119-121)
    float Dn[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int bc = 0; bc < 3; ++bc)
        Dn[a * 3 + bc] = D[a * 3 + bc] + dt * (C[a * 3 + bc] + C[a * 3 + 0] * D[0 * 3 + bc] +
                                               C[a * 3 + 1] * D[1 * 3 + bc] + C[a * 3 + 2] * D[2 * 3 + bc]);
#pragma unroll
    for (int e = 0; e < 9; ++e) D[e] = Dn[e];
    // x += dt v (src/three/mpm.js:122) in fixed point, clamped into the box
    const float s = dt * tc.invH * kFixedOne;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      // |dq| stays below 2^30 (a particle moves far less than 256 cells in a substep)
      long long qn = static_cast<long long>(q[a]) + __float2int_rn(fminf(fmaxf(s * v[a], -1.0e9f), 1.0e9f));
      if (tc.clamp) {
        qn = qn < (long long)tc.qlo[a] ? (long long)tc.qlo[a] : qn;
        qn = qn > (long long)tc.qhi[a] ? (long long)tc.qhi[a] : qn;
      } else {
        const long long hi = (static_cast<long long>(tc.dims[a]) - 1) << kFracBits;
        if (qn < 0 || qn > hi) flags |= 0x4u;
        qn = qn < 0 ? 0 : (qn > hi ? hi : qn);
      }
      q[a] = static_cast<unsigned>(qn);
    }
    // return map / stress for the next P2G (src/three/mpm.js:126-131)
    if constexpr (NEWTON) {
      const Sym3 B = cauchy_green_minus_identity(D);
      const int nt = learned_model(mt.model) ? series_terms_sq(sym_norm2(B)) : 0;
      if (nt > 0) {  // the series path of constitutive_update_t with the gated Johnson-Cook return
        const J2Trial tr = j2_trial_series(mt, B, nt);
        float dep = 0.f;
        const float f0 = jc_flow(mt, ep, 0.f, T);
        if (tr.q > f0) {
          const float u0 = fminf(1.f, fmaxf(0.f, 1.f - f0 / tr.q));
          const JcRefined r = jc_refine(mt, tr.q, tr.J, ep, T, dt, u0, c.gate_tol, c.learned_newton);
          dep = r.ok ? r.dep : jc_bisect(mt, tr.q, tr.J, ep, T, dt);
          // one shared atomic per group of converged lanes
          const unsigned act = __activemask(), acc = __ballot_sync(act, r.ok);
          if ((threadIdx.x & 31) == __ffs(act) - 1) {
            if (acc) atomicAdd(&gate[0], __popc(acc));
            if (act & ~acc) atomicAdd(&gate[1], __popc(act & ~acc));
          }
        }
        co = j2_finish(mt, tr, D, dep, V / m);
      } else {
        co = constitutive_update_t<AUX>(mt, D, ep, aux, T, V / m, true, dt, xp);
      }
    } else {
      co = constitutive_update_t<AUX>(mt, D, ep, aux, T, V / m, true, dt, xp);
    }
    ep += co.dep;
    T += co.dT;
    c.p.qx[home] = q[0]; c.p.qy[home] = q[1]; c.p.qz[home] = q[2];
#pragma unroll
    for (int e = 0; e < 9; ++e) c.p.Dc[e][home] = D[e];
    // v and C: the fused pass scatters the ones it just gathered and never reads the stored copies,
    // so it stores them only on the call's last substep (downloads, ledgers, frames, regularisation
    // and a later P2G of the stored state read them after the call); the gather-only pass always does
    if (PASS != kPassG2P2G || store_vc) {
      c.p.vx[home] = v[0]; c.p.vy[home] = v[1]; c.p.vz[home] = v[2];
#pragma unroll
      for (int e = 0; e < 9; ++e) c.p.Cc[e][home] = C[e];
    }
    if (c.has_plastic) c.p.ep[home] = ep;
    if (c.has_thermal) c.p.T[home] = T;
    if (AUX) c.p.aux[home] = aux;
    if (co.dep > 0.f && mt.heat_per_work > 0.f) atomicAdd(&work_acc, static_cast<double>(co.dT) * m / mt.heat_per_work);
  } else {
    // P2G of the stored state, and pinned particles (not moved, src/three/mpm.js:108)
    v[0] = c.p.vx[home]; v[1] = c.p.vy[home]; v[2] = c.p.vz[home];
#pragma unroll
    for (int e = 0; e < 9; ++e) C[e] = c.p.Cc[e][home];
    float Dc[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) Dc[e] = D[e];
    co = constitutive_update_t<AUX>(mt, Dc, ep, aux, T, V / m, false, 0.f, xp);
  }
  if (SCATTER) {
    // payload of the scatter: fraction t, m, m v, m C h, -4 V / h tau
    int nb[3];
    float t[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) stencil_axis(q[a], tc.dims[a], nb[a], t[a]);
    key = tile_key(sc, nb);
    if (PASS == kPassG2P2G) c.p.key[home] = key;
    const float mv[3] = {m * v[0], m * v[1], m * v[2]};
    const float mH = m * tc.H;
    float mC[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) mC[e] = mH * C[e];
    const float sv = -4.f * V * tc.invH;
    const float s6[6] = {sv * co.tau.xx, sv * co.tau.yy, sv * co.tau.zz, sv * co.tau.xy, sv * co.tau.xz, sv * co.tau.yz};
    const int l0 = nb[0] - (tc.tile[0] * kTile - 1), l1 = nb[1] - (tc.tile[1] * kTile - 1),
              l2 = nb[2] - (tc.tile[2] * kTile - 1);
    const bool in_w = l0 >= 0 && l0 <= kWinS - 3 && l1 >= 0 && l1 <= kWinS - 3 && l2 >= 0 && l2 <= kWinS - 3;
    if (in_w && !pinned) {
      const int bucket = (l2 * 6 + l1) * 6 + l0;
      // one shared atomic per bucket among the warp's converged lanes (particles of one cell share
      // buckets), each lane's rank from its position among them
      const unsigned act = __activemask();
      const unsigned peers = __match_any_sync(act, bucket);
      const int leader = __ffs(peers) - 1, lane = threadIdx.x & 31;
      int rank0 = 0;
      if (lane == leader) rank0 = atomicAdd(&hist[bucket], __popc(peers));
      const int rank = __shfl_sync(peers, rank0, leader) + __popc(peers & ((1u << lane) - 1u));
      meta[j] = static_cast<unsigned>(bucket) | (static_cast<unsigned>(rank) << 8);
      float2* P = pay + pay_slot(j);
      P[0 * kPayStride] = make_float2(t[0], t[1]);
      P[1 * kPayStride] = make_float2(t[2], m);
      P[2 * kPayStride] = make_float2(mv[0], mv[1]);
      P[3 * kPayStride] = make_float2(mv[2], HEAT ? m * T : 0.f);
      P[4 * kPayStride] = make_float2(mC[2], mC[5]);
      P[5 * kPayStride] = make_float2(mC[8], s6[4]);
      P[6 * kPayStride] = make_float2(s6[5], s6[2]);
      P[7 * kPayStride] = make_float2(mC[1], mC[4]);
      P[8 * kPayStride] = make_float2(mC[7], s6[3]);
      P[9 * kPayStride] = make_float2(mC[0], mC[3]);
      P[10 * kPayStride] = make_float2(mC[6], s6[0]);
      P[11 * kPayStride] = make_float2(s6[1], 0.f);
    } else {
      meta[j] = kMetaInvalid;
      if (!in_w) flags |= 0x10u;
      // copies scoped to this rare branch: the arrays passed to the out-of-line scatter would
      // otherwise live in local memory on every particle's path (3% of the fused pass)
      int nb_g[3];
      float t_g[3], mv_g[3], mC_g[9], s6_g[6];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        nb_g[a] = nb[a];
        t_g[a] = t[a];
        mv_g[a] = mv[a];
      }
#pragma unroll
      for (int e = 0; e < 9; ++e) mC_g[e] = mC[e];
#pragma unroll
      for (int e = 0; e < 6; ++e) s6_g[e] = s6[e];
      scatter_global(c, sc, tc, nxt, nb_g, t_g, m, mv_g, mC_g, s6_g, pinned, m * T);
    }
  }
  float wave, grad;
  cfl_terms<AUX>(mt, D, v, C, m, V, co.Jm1, aux, wave, grad);
  flags |= state_flags(v, D, co.tau, co.Jm1);
  flags_acc |= flags;
  wave_acc = fmaxf(wave_acc, wave);
  grad_acc = fmaxf(grad_acc, grad);
  return key;
}

// The learned Johnson-Cook return of one warp's particles. Every lane of the warp calls it; lanes
// with need set hold a trial stress above the initial flow stress. The network's guess (warp-wide
// tensor-core tiles), the refinement and gate, and the exact bisection for what the gate rejects,
// under one warp-uniform branch taken only by warps with such a lane. Inline: as an out-of-line
// call the particle state saved around it cost the pass 4% more with no return at all, and 5% more
// on an impact. gate[0] / gate[1] (shared memory) count the returns the gate accepted / sent to
// the bisection.
static __device__ __forceinline__ float learned_jc_return(const void* mlp_w, const float* mlp_params,
                                                      const MaterialDev& mt, float q, float J, float ep, float T,
                                                      float dt, bool need, float tol, int newton, unsigned* gate) {
  float x[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (need) jc_features(mt, q, J, ep, T, dt, x);
  const float u = surr::warp_predict_seq(static_cast<const surr::WeightsBf16*>(mlp_w), mlp_params, x[0], x[1], x[2],
                                         x[3], x[4], x[5], x[6], x[7]);
  JcRefined r{0.f, false};
  if (need) r = jc_refine(mt, q, J, ep, T, dt, u, tol, newton);
  const unsigned acc = __ballot_sync(0xffffffffu, need && r.ok), rej = __ballot_sync(0xffffffffu, need && !r.ok);
  if ((threadIdx.x & 31) == 0) {
    if (acc) atomicAdd(&gate[0], __popc(acc));
    if (rej) atomicAdd(&gate[1], __popc(rej));
  }
  if (need && !r.ok) r.dep = jc_bisect(mt, q, J, ep, T, dt);
  return r.dep;
}

// Phase A of the learned return mode (fused or gather-only pass; scenes without conduction and
// without the history laws). The same particle update as particle_phase_a, with the plastic
// increment of Johnson-Cook trial states (src/three/metal-plasticity.js:28-34) taken from the
// network: the warp evaluates it on the tensor cores for its lanes whose trial stress exceeds the
// initial flow stress, each such lane refines the prediction by Newton steps and keeps it if the
// consistency residual passes the gate (|g| <= gate_tol, i.e. the stress residual is at most
// gate_tol x the trial stress), and every other lane runs the exact bisection. Every lane of the
// warp calls it: lanes past the end of the round (live false) read the round's first particle,
// take part in the network evaluation and write nothing.
template <int PASS>
__device__ __forceinline__ unsigned particle_phase_a_learned(const Ctx& c, const SceneDev& sc, const TileCtx& tc,
                                                             const MaterialDev& mt_single, bool single,
                                                             const float4* vwin, bool live, unsigned home, unsigned j,
                                                             float dt, int nxt, float2* pay, unsigned* meta, int* hist,
                                                             float& wave_acc, float& grad_acc, unsigned& flags_acc,
                                                             double& work_acc, bool store_vc, unsigned* gate) {
  constexpr bool SCATTER = PASS != kPassG2P;
  static_assert(PASS != kPassP2G, "the learned mode changes only returns");
  unsigned key = 0xffffffffu;
  unsigned q[3] = {c.p.qx[home], c.p.qy[home], c.p.qz[home]};
  float D[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) D[e] = c.p.Dc[e][home];
  const float m = c.p.m[home], V = c.p.V[home];
  const MaterialDev& mt = single ? mt_single : c.mats[c.p.mat[home]];
  const bool pinned = c.has_pinned && c.p.pinned[home];
  float ep = c.has_plastic ? c.p.ep[home] : 0.f;
  float T = c.has_thermal ? c.p.T[home] : 0.f;
  float aux = 0.f;
  float v[3], C[9];
  unsigned flags = 0;
  const bool moving = !pinned;
  J2Trial tr{};
  bool series = false;
  if (moving) {
    int b[3];
    float t[3], w[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      stencil_axis(q[a], tc.dims[a], b[a], t[a]);
      bspline_weights(t[a], w[a]);
    }
    const int l0 = b[0] - tc.tile[0] * kTile, l1 = b[1] - tc.tile[1] * kTile, l2 = b[2] - tc.tile[2] * kTile;
    const bool in_g = l0 >= 0 && l0 <= kWinG - 3 && l1 >= 0 && l1 <= kWinG - 3 && l2 >= 0 && l2 <= kWinG - 3;
    if (!in_g) flags |= 0x20u;
    float acc12[12];
    if (in_g) {
      const float4* win = &vwin[(l2 * kWinG + l1) * kWinG + l0];
      gather27([&](int kz, int ky, int kx) { return win[(kz * kWinG + ky) * kWinG + kx]; }, t, w, acc12);
    } else {
      const Gather12 g = gather_global(c.g.vel + tc.node_base + ((long long)b[2] * tc.gdim[1] + b[1]) * tc.gdim[0] + b[0],
                                       tc.gdim[0], (long long)tc.gdim[0] * tc.gdim[1], t[0], t[1], t[2]);
#pragma unroll
      for (int e = 0; e < 12; ++e) acc12[e] = g.v[e];
    }
    const float s4 = 4.f * tc.invH;
    v[0] = acc12[0]; v[1] = acc12[1]; v[2] = acc12[2];
#pragma unroll
    for (int e = 0; e < 9; ++e) C[e] = acc12[3 + e] * s4;
    float Dn[9];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int bc = 0; bc < 3; ++bc)
        Dn[a * 3 + bc] = D[a * 3 + bc] + dt * (C[a * 3 + bc] + C[a * 3 + 0] * D[0 * 3 + bc] +
                                               C[a * 3 + 1] * D[1 * 3 + bc] + C[a * 3 + 2] * D[2 * 3 + bc]);
#pragma unroll
    for (int e = 0; e < 9; ++e) D[e] = Dn[e];
    const float s = dt * tc.invH * kFixedOne;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      long long qn = static_cast<long long>(q[a]) + __float2int_rn(fminf(fmaxf(s * v[a], -1.0e9f), 1.0e9f));
      if (tc.clamp) {
        qn = qn < (long long)tc.qlo[a] ? (long long)tc.qlo[a] : qn;
        qn = qn > (long long)tc.qhi[a] ? (long long)tc.qhi[a] : qn;
      } else {
        const long long hi = (static_cast<long long>(tc.dims[a]) - 1) << kFracBits;
        if (qn < 0 || qn > hi) flags |= 0x4u;
        qn = qn < 0 ? 0 : (qn > hi ? hi : qn);
      }
      q[a] = static_cast<unsigned>(qn);
    }
    // trial invariants of the J2-type laws on the series path
    if (mt.model >= 4 && mt.model != 8 && mt.model != 9) {
      const Sym3 B = cauchy_green_minus_identity(D);
      const int nt = series_terms_sq(sym_norm2(B));
      if (nt > 0) {
        tr = j2_trial_series(mt, B, nt);
        series = true;
      }
    }
  } else {
    v[0] = c.p.vx[home]; v[1] = c.p.vy[home]; v[2] = c.p.vz[home];
#pragma unroll
    for (int e = 0; e < 9; ++e) C[e] = c.p.Cc[e][home];
  }
  // the warp's learned return (every lane arrives here)
  const bool need = live && series && learned_model(mt.model) && tr.q > jc_flow(mt, ep, 0.f, T);
  float dep_learned = 0.f;
  if (__any_sync(0xffffffffu, need))
    dep_learned = learned_jc_return(c.mlp_w, c.mlp_params, mt, tr.q, tr.J, ep, T, dt, need, c.gate_tol,
                                    c.learned_newton, gate);
  ConstitutiveOut co;
  if (moving) {
    if (series) {
      float dep = 0.f;
      if (need) {  // a Johnson-Cook trial stress above the initial flow stress
        dep = dep_learned;
      } else if (!learned_model(mt.model)) {  // the other J2-type laws (a Johnson-Cook state below yield: 0)
        dep = plastic_increment(mt, tr.q, tr.J, ep, T, dt);
      }
      co = j2_finish(mt, tr, D, dep, V / m);
    } else {
      co = constitutive_update_t<false>(mt, D, ep, aux, T, V / m, true, dt);
    }
    ep += co.dep;
    T += co.dT;
    if (live) {
      c.p.qx[home] = q[0]; c.p.qy[home] = q[1]; c.p.qz[home] = q[2];
#pragma unroll
      for (int e = 0; e < 9; ++e) c.p.Dc[e][home] = D[e];
      if (PASS != kPassG2P2G || store_vc) {
        c.p.vx[home] = v[0]; c.p.vy[home] = v[1]; c.p.vz[home] = v[2];
#pragma unroll
        for (int e = 0; e < 9; ++e) c.p.Cc[e][home] = C[e];
      }
      if (c.has_plastic) c.p.ep[home] = ep;
      if (c.has_thermal) c.p.T[home] = T;
      if (co.dep > 0.f && mt.heat_per_work > 0.f) atomicAdd(&work_acc, static_cast<double>(co.dT) * m / mt.heat_per_work);
    }
  } else {
    float Dc[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) Dc[e] = D[e];
    co = constitutive_update_t<false>(mt, Dc, ep, aux, T, V / m, false, 0.f);
  }
  if (!live) return key;
  if (SCATTER) {
    int nb[3];
    float t[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) stencil_axis(q[a], tc.dims[a], nb[a], t[a]);
    key = tile_key(sc, nb);
    if (PASS == kPassG2P2G) c.p.key[home] = key;
    const float mv[3] = {m * v[0], m * v[1], m * v[2]};
    const float mH = m * tc.H;
    float mC[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) mC[e] = mH * C[e];
    const float sv = -4.f * V * tc.invH;
    const float s6[6] = {sv * co.tau.xx, sv * co.tau.yy, sv * co.tau.zz, sv * co.tau.xy, sv * co.tau.xz, sv * co.tau.yz};
    const int l0 = nb[0] - (tc.tile[0] * kTile - 1), l1 = nb[1] - (tc.tile[1] * kTile - 1),
              l2 = nb[2] - (tc.tile[2] * kTile - 1);
    const bool in_w = l0 >= 0 && l0 <= kWinS - 3 && l1 >= 0 && l1 <= kWinS - 3 && l2 >= 0 && l2 <= kWinS - 3;
    if (in_w && !pinned) {
      const int bucket = (l2 * 6 + l1) * 6 + l0;
      const unsigned act = __activemask();
      const unsigned peers = __match_any_sync(act, bucket);
      const int leader = __ffs(peers) - 1, lane = threadIdx.x & 31;
      int rank0 = 0;
      if (lane == leader) rank0 = atomicAdd(&hist[bucket], __popc(peers));
      const int rank = __shfl_sync(peers, rank0, leader) + __popc(peers & ((1u << lane) - 1u));
      meta[j] = static_cast<unsigned>(bucket) | (static_cast<unsigned>(rank) << 8);
      float2* P = pay + pay_slot(j);
      P[0 * kPayStride] = make_float2(t[0], t[1]);
      P[1 * kPayStride] = make_float2(t[2], m);
      P[2 * kPayStride] = make_float2(mv[0], mv[1]);
      P[3 * kPayStride] = make_float2(mv[2], 0.f);
      P[4 * kPayStride] = make_float2(mC[2], mC[5]);
      P[5 * kPayStride] = make_float2(mC[8], s6[4]);
      P[6 * kPayStride] = make_float2(s6[5], s6[2]);
      P[7 * kPayStride] = make_float2(mC[1], mC[4]);
      P[8 * kPayStride] = make_float2(mC[7], s6[3]);
      P[9 * kPayStride] = make_float2(mC[0], mC[3]);
      P[10 * kPayStride] = make_float2(mC[6], s6[0]);
      P[11 * kPayStride] = make_float2(s6[1], 0.f);
    } else {
      meta[j] = kMetaInvalid;
      if (!in_w) flags |= 0x10u;
      // copies scoped to this rare branch: the arrays passed to the out-of-line scatter would
      // otherwise live in local memory on every particle's path
      int nb_g[3];
      float t_g[3], mv_g[3], mC_g[9], s6_g[6];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        nb_g[a] = nb[a];
        t_g[a] = t[a];
        mv_g[a] = mv[a];
      }
#pragma unroll
      for (int e = 0; e < 9; ++e) mC_g[e] = mC[e];
#pragma unroll
      for (int e = 0; e < 6; ++e) s6_g[e] = s6[e];
      scatter_global(c, sc, tc, nxt, nb_g, t_g, m, mv_g, mC_g, s6_g, pinned, 0.f);
    }
  }
  float wave, grad;
  cfl_terms<false>(mt, D, v, C, m, V, co.Jm1, aux, wave, grad);
  flags |= state_flags(v, D, co.tau, co.Jm1);
  flags_acc |= flags;
  wave_acc = fmaxf(wave_acc, wave);
  grad_acc = fmaxf(grad_acc, grad);
  return key;
}

// L2 prefetch of the particle state a claimed tile will read. Between physical re-sorts a tile's
// particles keep the contiguous home range the last re-sort gave them (apart from the few that
// changed tiles since), and the tile's perm lists them in about that order; one perm entry from the
// middle places the range, and one bulk prefetch per state array covers it with a margin. Only a
// hint: the range is clipped to the live particles and a wrong guess costs bandwidth, not results.
template <bool AUX>
__device__ __forceinline__ void prefetch_tile_state(const Ctx& c, uint4 it) {
  const long long cnt = it.z;
  if (cnt == 0) return;
  const long long mid = c.p.perm[it.y + it.z / 2];
  const long long lo = max(0ll, mid - (3 * cnt) / 4 - 32), hi = min(static_cast<long long>(c.n), mid + (3 * cnt) / 4 + 32);
  if (hi <= lo) return;
  auto pf = [&](const void* base, int esize) {
    const unsigned long long a = (reinterpret_cast<unsigned long long>(base) + lo * esize) & ~15ull;
    const unsigned long long b = (reinterpret_cast<unsigned long long>(base) + hi * esize + 15) & ~15ull;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(static_cast<unsigned>(b - a)) : "memory");
  };
  pf(c.p.qx, 4);
  pf(c.p.qy, 4);
  pf(c.p.qz, 4);
#pragma unroll
  for (int e = 0; e < 9; ++e) pf(c.p.Dc[e], 4);
  pf(c.p.m, 4);
  pf(c.p.V, 4);
  if (c.has_plastic) pf(c.p.ep, 4);
  if (c.has_thermal) pf(c.p.T, 4);
  if (AUX) pf(c.p.aux, 4);
  if (!c.single_material && !c.scene_material) pf(c.p.mat, 2);
  if (c.has_pinned) pf(c.p.pinned, 1);
}

// JC: 0 the exact return map; 1 and 2 the gated Johnson-Cook returns (1 from the network's guess,
// warp-collective phase A; 2 from the initial flow stress, the plain phase A with the gated
// return), scenes without conduction and without the history laws.
template <int PASS, bool HEAT, bool AUX, int JC = 0>
__global__ void __launch_bounds__(kBlock, 2) k_particles(const __grid_constant__ Ctx c) {
  static_assert(JC == 0 || (!HEAT && !AUX && PASS != kPassP2G), "gated instances: no conduction, no history laws");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PartSmem& sm = *reinterpret_cast<PartSmem*>(smem_raw);
  constexpr bool SCATTER = PASS != kPassG2P;
  constexpr bool GATHER = PASS != kPassP2G;
  Ctrl* ct = c.ctrl;
  if (PASS == kPassG2P2G && blockIdx.x == 0 && threadIdx.x == 0) {  // for the sort that follows
    ct->sort_list = ct->step_index & 1u;
    ct->sort_active = ct->done ? 0u : 1u;
  }
  if (PASS != kPassP2G && ct->done) return;
  const unsigned k = ct->step_index;
  const bool store_vc = ct->last_substep != 0u;
  // lists: the P2G pass reads the list its sort just wrote (k & 1) and scatters into acc[k & 1];
  // a substep (after k_begin advanced k) reads list (k - 1) & 1 and scatters into acc[k & 1]
  const int lst = PASS == kPassP2G ? (k & 1) : ((k - 1) & 1);
  const int nxt = k & 1;
  const bool use_tma = GATHER && c.use_tma;
  if (SCATTER) {
    for (int i = threadIdx.x; i < kChannels * kWinSNodes; i += kBlock) sm.acc[i] = 0.f;
    for (int i = threadIdx.x; i < kBuckets; i += kBlock) sm.hist[i] = 0;
  }
  if (threadIdx.x == 0) {
    mbar_init(&sm.mbar[0], 1);
    mbar_init(&sm.mbar[1], 1);
    fence_barrier_init();
    sm.abort_flag = 0;
    sm.gate[0] = sm.gate[1] = 0u;
    sm.tma_phase[0] = sm.tma_phase[1] = 0u;
    sm.work_sum = 0.0;
    sm.mt_row = -1;
    sm.pf_ok = 0;
    const unsigned idx = atomicAdd(&ct->work_next, 1u);
    sm.item[0] = idx < ct->work_count[lst] ? c.s.work[lst][idx] : make_uint4(0xffffffffu, 0, 0, 0);
    if (use_tma && sm.item[0].x != 0xffffffffu) {
      const uint4 it = sm.item[0];
      const SceneDev& sc = c.scenes[it.w];
      const int lt = static_cast<int>(it.x) - sc.tile_base;
      mbar_arrive_expect_tx(&sm.mbar[0], sizeof(sm.vwin[0]));
      tma_load_4d(sm.vwin[0], static_cast<const char*>(c.tmaps) + 128 * it.w, 0, (lt % sc.tiles[0]) * kTile,
                  ((lt / sc.tiles[0]) % sc.tiles[1]) * kTile, (lt / (sc.tiles[0] * sc.tiles[1])) * kTile, &sm.mbar[0]);
    }
  }
  int cb = 0;
  while (true) {
    __syncthreads();
    const uint4 it = sm.item[cb];
    if (it.x == 0xffffffffu) break;
    if (threadIdx.x == 0) {
      if (use_tma) {
        const unsigned ph = sm.tma_phase[cb];
        if (!mbar_wait_bounded(&sm.mbar[cb], ph)) {
          atomicOr(&ct->status, 0x8u);
          mbar_wait_bounded(&sm.mbar[cb], ph);  // a second bounded chance for the copy in flight
          sm.abort_flag = 1;
        }
        sm.tma_phase[cb] ^= 1u;
      }
    }
    // The next work item is claimed, and its velocity window requested, by thread 0 after phase A
    // of this tile's first round, so the two dependent global round trips overlap other warps' work.
    auto prefetch_next = [&]() {
      const unsigned idx = atomicAdd(&ct->work_next, 1u);
      const uint4 nx = idx < ct->work_count[lst] ? c.s.work[lst][idx] : make_uint4(0xffffffffu, 0, 0, 0);
      sm.item[cb ^ 1] = nx;
      if (use_tma && nx.x != 0xffffffffu && !sm.abort_flag) {
        const SceneDev& sn = c.scenes[nx.w];
        const int lt = static_cast<int>(nx.x) - sn.tile_base;
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(&sm.mbar[cb ^ 1], sizeof(sm.vwin[0]));
        tma_load_4d(sm.vwin[cb ^ 1], static_cast<const char*>(c.tmaps) + 128 * nx.w, 0, (lt % sn.tiles[0]) * kTile,
                    ((lt / sn.tiles[0]) % sn.tiles[1]) * kTile, (lt / (sn.tiles[0] * sn.tiles[1])) * kTile,
                    &sm.mbar[cb ^ 1]);
      }
      if (nx.x != 0xffffffffu) prefetch_tile_state<AUX>(c, nx);
    };
    const int scene = static_cast<int>(it.w);
    const SceneDev& sc = c.scenes[scene];
    if (threadIdx.x == 0) {  // per-tile constants, computed once and read from shared memory
      TileCtx tl;
      const int lt = static_cast<int>(it.x) - sc.tile_base;
      tl.tile[0] = lt % sc.tiles[0];
      tl.tile[1] = (lt / sc.tiles[0]) % sc.tiles[1];
      tl.tile[2] = lt / (sc.tiles[0] * sc.tiles[1]);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        tl.dims[a] = sc.dims[a];
        tl.gdim[a] = sc.gdim[a];
        tl.qlo[a] = sc.qlo[a];
        tl.qhi[a] = sc.qhi[a];
      }
      tl.node_base = sc.node_base;
      tl.H = sc.H;
      tl.invH = sc.invH;
      tl.clamp = sc.clamp;
      tl.mat = sc.mat_base;
      sm.tc = tl;
    }
    // the material row of a single-material handle or of the tile's scene in a batch, copied word
    // by word by the whole block, and only when it changes (every tile of a one-scene handle shares
    // it; a batch's tiles come scene by scene)
    const int mt_row = sm.mt_row;
    if ((c.single_material || c.scene_material) && sc.mat_base != mt_row) {
      static_assert(sizeof(MaterialDev) % 4 == 0, "word copy");
      const unsigned* src = reinterpret_cast<const unsigned*>(c.mats + sc.mat_base);
      unsigned* dst = reinterpret_cast<unsigned*>(&sm.mt);
      for (int i = threadIdx.x; i < static_cast<int>(sizeof(MaterialDev) / 4); i += kBlock) dst[i] = src[i];
      __syncthreads();
      if (threadIdx.x == 0) sm.mt_row = sc.mat_base;
    }
    __syncthreads();
    if (sm.abort_flag) return;
    if (GATHER && !use_tma) {
      const TileCtx& tl = sm.tc;
      for (int i = threadIdx.x; i < kWinG * kWinG * kWinG; i += kBlock) {
        const int x = tl.tile[0] * kTile + i % kWinG, y = tl.tile[1] * kTile + (i / kWinG) % kWinG,
                  z = tl.tile[2] * kTile + i / (kWinG * kWinG);
        sm.vwin[cb][i] = c.g.vel[tl.node_base + ((long long)z * tl.gdim[1] + y) * tl.gdim[0] + x];
      }
      __syncthreads();
    }
    const TileCtx& tc = sm.tc;
    const float dt = GATHER ? c.dt_scene[scene] : 0.f;
    const bool single = c.single_material != 0 || c.scene_material != 0;
    float wave_acc = 0.f, grad_acc = 0.f;
    unsigned flags_acc = 0;
    for (unsigned r0 = 0; r0 < sm.item[cb].z; r0 += kCap) {
      const unsigned nround = min(static_cast<unsigned>(kCap), sm.item[cb].z - r0);
      // ---- phase A: one thread per particle (the bucket histogram is zero: cleared at the start
      // and by each round's scan) ----
      for (unsigned jj = 0; jj < nround; jj += kBlock) {
        const unsigned j = jj + threadIdx.x;
        unsigned key = 0xffffffffu;
        if constexpr (JC == 1) {
          // every lane of a warp with a live particle takes part in its network evaluation (warps
          // past the end of the round skip as a whole)
          if (jj + (threadIdx.x & ~31u) >= nround) continue;
          const bool live = j < nround;
          const unsigned home = !live ? c.p.perm[it.y + r0]
                                      : (r0 == 0 && sm.pf_ok && jj < kPf * kBlock) ? sm.pfs[jj + threadIdx.x]
                                                                                 : c.p.perm[it.y + r0 + j];
          key = particle_phase_a_learned<PASS>(c, sc, tc, sm.mt, single, sm.vwin[cb], live, home, j, dt, nxt, sm.pay,
                                               sm.meta, sm.hist, wave_acc, grad_acc, flags_acc, sm.work_sum, store_vc,
                                               sm.gate);
        } else if (j < nround) {
          const unsigned home = (r0 == 0 && sm.pf_ok && jj < kPf * kBlock) ? sm.pfs[jj + threadIdx.x] : c.p.perm[sm.item[cb].y + r0 + j];
          key = particle_phase_a<PASS, HEAT, AUX, JC == 2>(c, sc, tc, sm.mt, single, sm.vwin[cb], home, j, dt, nxt,
                                                           sm.pay, sm.meta, sm.hist, wave_acc, grad_acc, flags_acc,
                                                           sm.work_sum, store_vc, sm.gate);
        }
        if (PASS == kPassG2P2G) count_key(c, key);
      }
      if (!SCATTER && r0 == 0 && threadIdx.x == 0) prefetch_next();
      if (SCATTER) {
        __syncthreads();
        scan_buckets(sm);
        __syncthreads();
        for (unsigned j = threadIdx.x; j < nround; j += kBlock) {
          const unsigned mm = sm.meta[j];
          if (!(mm & kMetaInvalid)) sm.sidx[sm.bstart[mm & 0xffu] + (mm >> 8)] = static_cast<unsigned short>(j);
        }
        __syncthreads();
        // ---- phase B: one thread per (non-empty bucket, z layer); the last thread claims the next
        // tile meanwhile (a full tile has about 3 x 64 tasks, so it rarely has one)
        if (r0 == 0 && threadIdx.x == kBlock - 1) prefetch_next();
        const int nbk = sm.nbuckets;
        for (int task = threadIdx.x; task < 3 * nbk; task += kBlock) {
          const int kz = task / nbk;
          bucket_layer<HEAT>(sm, sm.blist[task - kz * nbk], kz);
        }
        __syncthreads();
        if (r0 == 0) {  // perm of the next tile's first round, consumed there
          const uint4 nx = sm.item[cb ^ 1];
          const bool ok = nx.x != 0xffffffffu;
          if (threadIdx.x == 0) sm.pf_ok = ok;
          if (ok) {
#pragma unroll
            for (int k = 0; k < kPf; ++k) {
              const unsigned j = k * kBlock + threadIdx.x;
              sm.pfs[j] = j < nx.z ? c.p.perm[nx.y + j] : 0u;
            }
          }
        }
      }
    }
    block_reduce_item(c, scene, wave_acc, grad_acc, flags_acc, sm.red);
    __syncthreads();
    if (SCATTER) flush_window(c, sc, sm, nxt, tc.tile);
    cb ^= 1;
  }
  if (JC != 0 && threadIdx.x == 0) {  // gate counts: one atomic each per CTA (the loop ended at a barrier)
    if (sm.gate[0]) atomicAdd(&c.gate_counts[0], sm.gate[0]);
    if (sm.gate[1]) atomicAdd(&c.gate_counts[1], sm.gate[1]);
  }
  // heat from plastic work: one FP64 atomic per CTA (the loop ended at a barrier)
  if (GATHER && threadIdx.x == 0 && sm.work_sum != 0.0) atomicAdd(&ct->plastic_work, sm.work_sum);
}

// ---------------------------------------------------------------------------------------------
// Warp-specialised particle pass (P2G and G2P2G): one CTA of two 256-thread groups per SM.
//   producer group (warps 0-7): claims tiles, waits for their TMA velocity window, runs phase A
//     (one thread per particle) into one of two stage buffers (payload, bucket keys, histogram)
//   consumer group (warps 8-15): scans the buckets of a finished stage, runs phase B (the register
//     accumulation per bucket and z layer) into the shared scatter window and flushes the window
//     to HBM after the last stage of a tile
// so phase A of one tile overlaps phase B of the previous one, and neither group waits at a
// CTA-wide barrier for the other's slowest thread. Stage hand-off uses mbarriers (full: producer
// -> consumer, empty: consumer -> producer) with bounded waits; a wait that gives up sets the
// timeout status and both groups leave through the same sentinel path.

constexpr int kWsGroup = 256;
constexpr int kWsThreads = 2 * kWsGroup;

struct StageInfo {
  TileCtx tc;
  int nround;
  int flush;     // last round of its tile: the consumer flushes the window after it
  int scene;
  int sentinel;  // no more stages
};

struct __align__(128) WsSmem {
  float4 vwin[2][kWinG * kWinG * kWinG];  // producer: double-buffered TMA destinations
  float2 pay[2][kPayRows * kPayStride];   // stage buffers
  unsigned meta[2][kCap];
  int hist[2][kBuckets];
  StageInfo info[2];
  float acc[kChannels * kWinSNodes];      // consumer: scatter window
  unsigned short sidx[kCap];
  int bstart[kBuckets + 1];
  unsigned short blist[kBuckets];
  int nbuckets;
  int wsum[kWsGroup / 32], wnz[kWsGroup / 32];  // per-warp bucket totals of the consumer scan
  StageInfo flush_info;                   // consumer copy of the stage it flushes
  unsigned long long tma_bar[2], full[2], empty[2];
  uint4 item[2];
  int abort_flag;                         // producer gave up (its TMA wait timed out)
  int consumer_exit;                      // consumer gave up waiting for a stage
  unsigned red[3 * (kWsGroup / 32)];
  double work_sum;  // heat from plastic work of the CTA's particles
  TileCtx tc;
  MaterialDev mt;
};

size_t ws_smem_bytes() { return sizeof(WsSmem); }

__device__ __forceinline__ void group_sync(int id) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(kWsGroup) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Per-tile CFL maxima and status flags over the producer group, then one atomic per tile.
__device__ __forceinline__ void group_reduce_item(const Ctx& c, int scene, float wave, float grad, unsigned flags,
                                                  unsigned* red, int tid) {
  const unsigned wb = __reduce_max_sync(0xffffffffu, fbits(wave));
  const unsigned gb = __reduce_max_sync(0xffffffffu, fbits(grad));
  const unsigned fl = __reduce_or_sync(0xffffffffu, flags);
  const int lane = tid & 31, wid = tid >> 5;
  if (lane == 0) {
    red[wid * 3 + 0] = wb;
    red[wid * 3 + 1] = gb;
    red[wid * 3 + 2] = fl;
  }
  group_sync(1);
  if (tid == 0) {
    unsigned w = 0, g = 0, f = 0;
    for (int k = 0; k < kWsGroup / 32; ++k) {
      w = max(w, red[k * 3 + 0]);
      g = max(g, red[k * 3 + 1]);
      f |= red[k * 3 + 2];
    }
    atomicMax(&c.wave_max[scene], w);
    atomicMax(&c.grad_max[scene], g);
    if (f) atomicOr(&c.ctrl->status, f);
  }
}

template <int PASS, bool HEAT, bool AUX>
__global__ void __launch_bounds__(kWsThreads, 1) k_particles_ws(const __grid_constant__ Ctx c) {
  static_assert(PASS != kPassG2P, "the warp-specialised pass always scatters");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  WsSmem& sm = *reinterpret_cast<WsSmem*>(smem_raw);
  constexpr bool GATHER = PASS != kPassP2G;
  Ctrl* ct = c.ctrl;
  if (PASS == kPassG2P2G && blockIdx.x == 0 && threadIdx.x == 0) {  // for the sort that follows
    ct->sort_list = ct->step_index & 1u;
    ct->sort_active = ct->done ? 0u : 1u;
  }
  if (PASS != kPassP2G && ct->done) return;
  const unsigned k = ct->step_index;
  const bool store_vc = ct->last_substep != 0u;
  const int lst = PASS == kPassP2G ? (k & 1) : ((k - 1) & 1);
  const int nxt = k & 1;
  const bool use_tma = GATHER && c.use_tma;
  for (int i = threadIdx.x; i < kChannels * kWinSNodes; i += kWsThreads) sm.acc[i] = 0.f;
  auto issue_window = [&](int buf, const uint4& it) {
    const SceneDev& sn = c.scenes[it.w];
    const int lt = static_cast<int>(it.x) - sn.tile_base;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&sm.tma_bar[buf], sizeof(sm.vwin[0]));
    tma_load_4d(sm.vwin[buf], static_cast<const char*>(c.tmaps) + 128 * it.w, 0, (lt % sn.tiles[0]) * kTile,
                ((lt / sn.tiles[0]) % sn.tiles[1]) * kTile, (lt / (sn.tiles[0] * sn.tiles[1])) * kTile,
                &sm.tma_bar[buf]);
  };
  if (threadIdx.x == 0) {
    for (int b = 0; b < 2; ++b) {
      mbar_init(&sm.tma_bar[b], 1);
      mbar_init(&sm.full[b], 1);
      mbar_init(&sm.empty[b], 1);
    }
    fence_barrier_init();
    sm.abort_flag = 0;
    sm.consumer_exit = 0;
    sm.work_sum = 0.0;
    const unsigned idx = atomicAdd(&ct->work_next, 1u);
    sm.item[0] = idx < ct->work_count[lst] ? c.s.work[lst][idx] : make_uint4(0xffffffffu, 0, 0, 0);
    if (use_tma && sm.item[0].x != 0xffffffffu) issue_window(0, sm.item[0]);
  }
  __syncthreads();
  if (threadIdx.x < kWsGroup) {
    // ================= producer =================
    const int tid = threadIdx.x;
    int s = 0, cb = 0;
    unsigned uses[2] = {0u, 0u}, pe[2] = {0u, 0u}, tph[2] = {0u, 0u};
    bool in_flight[2] = {tid == 0 && use_tma && sm.item[0].x != 0xffffffffu, false};  // thread 0's TMA copies
    const bool single = c.single_material != 0 || c.scene_material != 0;
    bool stop = false;
    while (!stop) {
      group_sync(1);
      const uint4 it = sm.item[cb];
      if (it.x == 0xffffffffu) break;
      const int scene = static_cast<int>(it.w);
      const SceneDev& sc = c.scenes[scene];
      if (tid == 0) {
        if (use_tma) {
          if (!mbar_wait_bounded(&sm.tma_bar[cb], tph[cb])) {
            atomicOr(&ct->status, 0x8u);
            mbar_wait_bounded(&sm.tma_bar[cb], tph[cb]);  // a second bounded chance for the copy in flight
            sm.abort_flag = 1;
          }
          tph[cb] ^= 1u;
          in_flight[cb] = false;
        }
        // claim the next tile now: its window streams in while this tile is processed (the other
        // window buffer was last read by this group's previous tile)
        const unsigned idx = atomicAdd(&ct->work_next, 1u);
        const uint4 nx = idx < ct->work_count[lst] ? c.s.work[lst][idx] : make_uint4(0xffffffffu, 0, 0, 0);
        sm.item[cb ^ 1] = nx;
        if (use_tma && nx.x != 0xffffffffu && !sm.abort_flag) {
          issue_window(cb ^ 1, nx);
          in_flight[cb ^ 1] = true;
        }
        TileCtx tl;
        const int lt = static_cast<int>(it.x) - sc.tile_base;
        tl.tile[0] = lt % sc.tiles[0];
        tl.tile[1] = (lt / sc.tiles[0]) % sc.tiles[1];
        tl.tile[2] = lt / (sc.tiles[0] * sc.tiles[1]);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          tl.dims[a] = sc.dims[a];
          tl.gdim[a] = sc.gdim[a];
          tl.qlo[a] = sc.qlo[a];
          tl.qhi[a] = sc.qhi[a];
        }
        tl.node_base = sc.node_base;
        tl.H = sc.H;
        tl.invH = sc.invH;
        tl.clamp = sc.clamp;
        tl.mat = sc.mat_base;
        sm.tc = tl;
        if (single) sm.mt = c.mats[sc.mat_base];
      }
      group_sync(1);
      if (sm.abort_flag) break;
      if (GATHER && !use_tma) {
        const TileCtx& tl = sm.tc;
        for (int i = tid; i < kWinG * kWinG * kWinG; i += kWsGroup) {
          const int x = tl.tile[0] * kTile + i % kWinG, y = tl.tile[1] * kTile + (i / kWinG) % kWinG,
                    z = tl.tile[2] * kTile + i / (kWinG * kWinG);
          sm.vwin[cb][i] = c.g.vel[tl.node_base + ((long long)z * tl.gdim[1] + y) * tl.gdim[0] + x];
        }
        group_sync(1);
      }
      const TileCtx& tc = sm.tc;
      const float dt = GATHER ? c.dt_scene[scene] : 0.f;
      float wave_acc = 0.f, grad_acc = 0.f;
      unsigned flags_acc = 0;
      for (unsigned r0 = 0; r0 < it.z; r0 += kCap) {
        const unsigned nround = min(static_cast<unsigned>(kCap), it.z - r0);
        // take stage buffer s once the consumer has finished with it
        if (tid == 0 && uses[s]) {
          if (!mbar_wait_bounded(&sm.empty[s], pe[s])) {
            atomicOr(&ct->status, 0x8u);
            sm.abort_flag = 1;
          }
          pe[s] ^= 1u;
        }
        group_sync(1);
        if (sm.abort_flag) {
          stop = true;
          break;
        }
        for (int i = tid; i < kBuckets; i += kWsGroup) sm.hist[s][i] = 0;
        group_sync(1);
        for (unsigned jj = 0; jj < nround; jj += kWsGroup) {
          const unsigned j = jj + tid;
          unsigned key = 0xffffffffu;
          if (j < nround) {
            const unsigned home = c.p.perm[it.y + r0 + j];
            key = particle_phase_a<PASS, HEAT, AUX>(c, sc, tc, sm.mt, single, sm.vwin[cb], home, j, dt, nxt, sm.pay[s],
                                         sm.meta[s], sm.hist[s], wave_acc, grad_acc, flags_acc, sm.work_sum, store_vc);
          }
          if (PASS == kPassG2P2G) count_key(c, key);
        }
        if (tid == 0) {
          StageInfo inf;
          inf.tc = tc;
          inf.nround = static_cast<int>(nround);
          inf.flush = (r0 + kCap >= it.z) ? 1 : 0;
          inf.scene = scene;
          inf.sentinel = 0;
          sm.info[s] = inf;
        }
        group_sync(1);
        if (tid == 0) {
          __threadfence_block();
          mbar_arrive(&sm.full[s]);
        }
        ++uses[s];
        s ^= 1;
      }
      if (stop) break;
      group_reduce_item(c, scene, wave_acc, grad_acc, flags_acc, sm.red, tid);
      cb ^= 1;
    }
    // sentinel stage: the consumer leaves after it. A group that stopped early first lets its own
    // window copy in flight land (bounded), so no TMA writes into the CTA's memory after it exits.
    if (tid == 0) {
      for (int b = 0; b < 2; ++b)
        if (in_flight[b] && !mbar_wait_bounded(&sm.tma_bar[b], tph[b])) atomicOr(&ct->status, 0x8u);
      bool ok = true;
      if (uses[s]) ok = mbar_wait_bounded(&sm.empty[s], pe[s]);
      if (!ok) atomicOr(&ct->status, 0x8u);
      sm.info[s].sentinel = 1;
      __threadfence_block();
      mbar_arrive(&sm.full[s]);
    }
  } else {
    // ================= consumer =================
    const int tb = threadIdx.x - kWsGroup;
    int s = 0;
    unsigned pf[2] = {0u, 0u};
    while (true) {
      if (tb == 0) {
        if (!mbar_wait_bounded(&sm.full[s], pf[s])) {
          atomicOr(&ct->status, 0x8u);
          sm.consumer_exit = 1;
        }
        pf[s] ^= 1u;
      }
      group_sync(2);
      if (sm.consumer_exit || sm.info[s].sentinel) break;
      scan_buckets_group<kWsGroup>(sm.hist[s], sm.bstart, sm.blist, &sm.nbuckets, sm.wsum, sm.wnz, tb, false,
                                   [] { group_sync(2); });
      group_sync(2);
      const int nround = sm.info[s].nround;
      for (int j = tb; j < nround; j += kWsGroup) {
        const unsigned mm = sm.meta[s][j];
        if (!(mm & kMetaInvalid)) sm.sidx[sm.bstart[mm & 0xffu] + (mm >> 8)] = static_cast<unsigned short>(j);
      }
      group_sync(2);
      const int nbk = sm.nbuckets;
      for (int task = tb; task < 3 * nbk; task += kWsGroup) {
        const int kz = task / nbk;
        bucket_layer_p<HEAT>(sm.pay[s], sm.sidx, sm.bstart, sm.acc, sm.blist[task - kz * nbk], kz);
      }
      group_sync(2);
      if (tb == 0) {
        sm.flush_info = sm.info[s];  // the producer may reuse the stage once it is released
        __threadfence_block();
        mbar_arrive(&sm.empty[s]);
      }
      group_sync(2);
      if (sm.flush_info.flush) {
        flush_window_p(c, c.scenes[sm.flush_info.scene], sm.acc, nxt, sm.flush_info.tc.tile, tb, kWsGroup);
        group_sync(2);
      }
      s ^= 1;
    }
  }
  // heat from plastic work: one FP64 atomic per CTA
  __syncthreads();
  if (GATHER && threadIdx.x == 0 && sm.work_sum != 0.0) atomicAdd(&ct->plastic_work, sm.work_sum);
}

template <int PASS, bool HEAT, bool AUX>
static void launch_pass_t(const Ctx& c, cudaStream_t st, int grid_blocks) {
  if constexpr (PASS != kPassP2G && !HEAT && !AUX) {
    if (c.learned == 1) {
      k_particles<PASS, false, false, 1><<<grid_blocks, kBlock, sizeof(PartSmem), st>>>(c);
      return;
    }
    if (c.learned == 2) {
      k_particles<PASS, false, false, 2><<<grid_blocks, kBlock, sizeof(PartSmem), st>>>(c);
      return;
    }
  }
  if (PASS != kPassG2P && c.ws_blocks > 0) {
    k_particles_ws<PASS == kPassG2P ? kPassG2P2G : PASS, HEAT, AUX><<<c.ws_blocks, kWsThreads, sizeof(WsSmem), st>>>(c);
    return;
  }
  k_particles<PASS, HEAT, AUX><<<grid_blocks, kBlock, sizeof(PartSmem), st>>>(c);
}

// The heat channel and the conduction gather are compiled only into the conducting instances, the
// history scalar of snow, sand and the pressure laws only into the instances for those materials.
template <int PASS>
static void launch_pass(const Ctx& c, cudaStream_t st, int grid_blocks) {
  if (c.conduct) {
    if (c.has_aux) launch_pass_t<PASS, true, true>(c, st, grid_blocks);
    else launch_pass_t<PASS, true, false>(c, st, grid_blocks);
  } else {
    if (c.has_aux) launch_pass_t<PASS, false, true>(c, st, grid_blocks);
    else launch_pass_t<PASS, false, false>(c, st, grid_blocks);
  }
}

void launch_p2g(const Ctx& c, cudaStream_t st, int grid_blocks) { launch_pass<kPassP2G>(c, st, grid_blocks); }

void launch_g2p2g(const Ctx& c, cudaStream_t st, int grid_blocks, bool scatter) {
  if (scatter)
    launch_pass<kPassG2P2G>(c, st, grid_blocks);
  else
    launch_pass<kPassG2P>(c, st, grid_blocks);
}

template <int PASS>
static int blocks_per_sm() {
  const int bytes = (int)sizeof(PartSmem);
  cudaFuncSetAttribute(k_particles<PASS, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_particles<PASS, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_particles<PASS, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_particles<PASS, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if constexpr (PASS != kPassP2G) {
    cudaFuncSetAttribute(k_particles<PASS, false, false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(k_particles<PASS, false, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  }
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_particles<PASS, false, false>, kBlock, sizeof(PartSmem));
  return n > 0 ? n : 1;
}

// Resident CTAs per SM of the warp-specialised pass (0: it cannot launch here).
int ws_blocks_per_sm() {
  int n0 = 0, n1 = 0;
  const int bytes = (int)sizeof(WsSmem);
  auto set = [&](const void* fn) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
  };
  if (!set((const void*)k_particles_ws<kPassP2G, false, false>) || !set((const void*)k_particles_ws<kPassG2P2G, false, false>) ||
      !set((const void*)k_particles_ws<kPassP2G, true, false>) || !set((const void*)k_particles_ws<kPassG2P2G, true, false>) ||
      !set((const void*)k_particles_ws<kPassP2G, false, true>) || !set((const void*)k_particles_ws<kPassG2P2G, false, true>) ||
      !set((const void*)k_particles_ws<kPassP2G, true, true>) || !set((const void*)k_particles_ws<kPassG2P2G, true, true>))
    return 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n0, k_particles_ws<kPassP2G, true, true>, kWsThreads, sizeof(WsSmem));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n1, k_particles_ws<kPassG2P2G, true, true>, kWsThreads, sizeof(WsSmem));
  return n0 < n1 ? n0 : n1;
}

int g2p2g_blocks_per_sm(bool scatter) { return scatter ? blocks_per_sm<kPassG2P2G>() : blocks_per_sm<kPassG2P>(); }

int p2g_blocks_per_sm() { return blocks_per_sm<kPassP2G>(); }


// Grid update over the active node tiles (src/three/mpm.js:89-102 with gravity on the grid).
__global__ void __launch_bounds__(256) k_grid_update(Ctx c) {
  Ctrl* ct = c.ctrl;
  if (ct->done) return;
  const unsigned k = ct->step_index;
  const int cur = (k - 1) & 1;
  const unsigned count = ct->active_count[cur];
  const int sub = threadIdx.x >> 6, lid = threadIdx.x & 63;
  for (unsigned ti = blockIdx.x * 4 + sub; ti < count; ti += gridDim.x * 4) {
    const unsigned tile = c.g.active[cur][ti];
    const int s = c.nscenes == 1 ? 0 : find_scene_by_node_tile(c.scenes, c.nscenes, static_cast<int>(tile));
    const SceneDev& sc = c.scenes[s];
    const int lt = static_cast<int>(tile) - sc.node_tile_base;
    const int ntx = lt % sc.ntiles[0], nty = (lt / sc.ntiles[0]) % sc.ntiles[1], ntz = lt / (sc.ntiles[0] * sc.ntiles[1]);
    const int x = ntx * 4 + (lid & 3), y = nty * 4 + ((lid >> 2) & 3), z = ntz * 4 + (lid >> 4);
    const long long node = sc.node_base + ((long long)z * sc.gdim[1] + y) * sc.gdim[0] + x;
    const float4 a0 = c.g.acc0[cur][node];
    const float4 a1 = c.g.acc1[cur][node];
    float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
    if (a0.x > sc.mass_eps) {
      const float dt = c.dt_scene[s];
      const float inv = 1.f / a0.x;
      float v[3] = {(a0.y + dt * (a1.x + a0.x * sc.gravity[0])) * inv,
                    (a0.z + dt * (a1.y + a0.x * sc.gravity[1])) * inv,
                    (a0.w + dt * (a1.z + a0.x * sc.gravity[2])) * inv};
      const int idx[3] = {x, y, z};
      const bool all_zero = (a1.w > 0.f) || (sc.sticky && y <= sc.wall_lo[1]);
#pragma unroll
      for (int a = 0; a < 3; ++a)
        if (all_zero || (idx[a] <= sc.wall_lo[a] && v[a] < 0.f) || (idx[a] >= sc.wall_hi[a] && v[a] > 0.f)) v[a] = 0.f;
      out = make_float4(v[0], v[1], v[2], a0.x);
    }
    c.g.vel[node] = out;
    c.g.acc0[cur][node] = make_float4(0.f, 0.f, 0.f, 0.f);
    c.g.acc1[cur][node] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c.conduct) {  // node temperature and mass for the conduction pass
      const bool has = a0.x > sc.mass_eps;
      c.g.tnode[node] = has ? c.g.heat[cur][node] / a0.x : 0.f;
      c.g.mnode[node] = has ? a0.x : 0.f;
      c.g.heat[cur][node] = 0.f;
      if (lid == 0) c.g.tile_epoch[tile] = k;
    }
    if (lid == 0) c.g.tile_flag[tile] = 0u;
  }
}

// Grid heat conduction (explicit, between face-neighbour nodes that both hold mass this substep):
// Q_ij = G_ij (T_j - T_i), G_ij = k h dt min(1, min(m_i, m_j) / (rho h^3)); dT_i = sum_j Q_ij /
// (m_i cp), written to the node's fourth velocity channel for the gather. G is symmetric, so the
// nodes' heat sum m cp T is unchanged; the mass factor keeps partly filled nodes under the same
// stability limit as full ones (6 k dt / (rho cp h^2) < 1). A neighbour counts only if its node
// tile was updated in this substep (its stored mass and temperature are current).
__global__ void __launch_bounds__(256) k_conduct(Ctx c) {
  Ctrl* ct = c.ctrl;
  if (ct->done) return;
  const unsigned k = ct->step_index;
  const int cur = (k - 1) & 1;
  const unsigned count = ct->active_count[cur];
  const int sub = threadIdx.x >> 6, lid = threadIdx.x & 63;
  for (unsigned ti = blockIdx.x * 4 + sub; ti < count; ti += gridDim.x * 4) {
    const unsigned tile = c.g.active[cur][ti];
    const int s = c.nscenes == 1 ? 0 : find_scene_by_node_tile(c.scenes, c.nscenes, static_cast<int>(tile));
    const SceneDev& sc = c.scenes[s];
    const int lt = static_cast<int>(tile) - sc.node_tile_base;
    const int ntx = lt % sc.ntiles[0], nty = (lt / sc.ntiles[0]) % sc.ntiles[1], ntz = lt / (sc.ntiles[0] * sc.ntiles[1]);
    const int x = ntx * 4 + (lid & 3), y = nty * 4 + ((lid >> 2) & 3), z = ntz * 4 + (lid >> 4);
    const long long node = sc.node_base + ((long long)z * sc.gdim[1] + y) * sc.gdim[0] + x;
    const float mi = c.g.mnode[node];
    float dT = 0.f;
    if (sc.cond_G > 0.f && mi > sc.mass_eps) {
      const float Ti = c.g.tnode[node];
      const float g0 = sc.cond_G * c.dt_scene[s];
      float q = 0.f;
      const int xyz[3] = {x, y, z};
      const long long stride[3] = {1, sc.gdim[0], (long long)sc.gdim[0] * sc.gdim[1]};
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int d = -1; d <= 1; d += 2) {
          const int p = xyz[a] + d;
          if (p < 0 || p >= sc.gdim[a]) continue;
          int nt[3] = {x >> 2, y >> 2, z >> 2};
          nt[a] = p >> 2;
          const unsigned jt = static_cast<unsigned>(sc.node_tile_base + (nt[2] * sc.ntiles[1] + nt[1]) * sc.ntiles[0] + nt[0]);
          if (c.g.tile_epoch[jt] != k) continue;
          const long long nj = node + d * stride[a];
          const float mj = c.g.mnode[nj];
          if (!(mj > sc.mass_eps)) continue;
          q += g0 * fminf(1.f, fminf(mi, mj) * sc.cond_inv_mfull) * (c.g.tnode[nj] - Ti);
        }
      dT = q * sc.cond_inv_cp / mi;
    }
    c.g.vel[node].w = dT;
  }
}

void launch_conduct(const Ctx& c, cudaStream_t st, int grid_blocks) { k_conduct<<<grid_blocks, 256, 0, st>>>(c); }

// ---------------------------------------------------------------------------------------------
// Slab decomposition of one domain along z. Scenes s and s+1 (or two ranks' scenes) hold the same
// `planes` node planes: the top planes of s are the bottom planes of s+1. After each scatter (the
// fresh grid is acc[step_index & 1]) both copies of a shared node must hold the sum of both
// slabs' contributions, so both grid updates give the same velocity there; a copy is written only
// where its node tile is active this substep (inactive tiles are never read by the grid update,
// which would also never clear them).

__device__ __forceinline__ bool node_active(const Ctx& c, const SceneDev& sc, int x, int y, int z) {
  const unsigned tile = sc.node_tile_base + ((z >> 2) * sc.ntiles[1] + (y >> 2)) * sc.ntiles[0] + (x >> 2);
  return c.g.tile_flag[tile] != 0u;
}

__global__ void k_halo_sum(Ctx c, int planes) {
  if (c.ctrl->done) return;
  const int par = c.ctrl->step_index & 1;
  for (int s = 0; s + 1 < c.nscenes; ++s) {
    const SceneDev& lo = c.scenes[s];
    const SceneDev& hi = c.scenes[s + 1];
    const long long per = (long long)lo.gdim[0] * lo.gdim[1];
    const long long total = per * planes;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
      const int zr = static_cast<int>(i / per);
      const int rem = static_cast<int>(i - (long long)zr * per);
      const int y = rem / lo.gdim[0], x = rem - y * lo.gdim[0];
      const int zl = lo.dims[2] - planes + zr;
      const long long nl = lo.node_base + ((long long)zl * lo.gdim[1] + y) * lo.gdim[0] + x;
      const long long nh = hi.node_base + ((long long)zr * hi.gdim[1] + y) * hi.gdim[0] + x;
      const bool al = node_active(c, lo, x, y, zl), ah = node_active(c, hi, x, y, zr);
      if (!al && !ah) continue;
      const float4 a0 = c.g.acc0[par][nl], b0 = c.g.acc0[par][nh];
      const float4 a1 = c.g.acc1[par][nl], b1 = c.g.acc1[par][nh];
      const float4 s0 = make_float4(a0.x + b0.x, a0.y + b0.y, a0.z + b0.z, a0.w + b0.w);
      const float4 s1 = make_float4(a1.x + b1.x, a1.y + b1.y, a1.z + b1.z, a1.w + b1.w);
      if (al) { c.g.acc0[par][nl] = s0; c.g.acc1[par][nl] = s1; }
      if (ah) { c.g.acc0[par][nh] = s0; c.g.acc1[par][nh] = s1; }
      if (c.conduct) {
        const float hs = c.g.heat[par][nl] + c.g.heat[par][nh];
        if (al) c.g.heat[par][nl] = hs;
        if (ah) c.g.heat[par][nh] = hs;
      }
    }
  }
}

void launch_halo_sum(const Ctx& c, cudaStream_t st, int planes) {
  if (c.nscenes < 2 || planes <= 0) return;
  k_halo_sum<<<1184, 256, 0, st>>>(c, planes);
}

__global__ void k_halo_copy(Ctx c, int side, int planes, float* out, const float* in) {
  if (c.ctrl->done) return;
  const int par = c.ctrl->step_index & 1;
  const SceneDev& sc = c.scenes[0];
  const long long per = (long long)sc.gdim[0] * sc.gdim[1];
  const long long total = per * planes;
  const int z0 = side == 0 ? 0 : sc.dims[2] - planes;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int zr = static_cast<int>(i / per);
    const int rem = static_cast<int>(i - (long long)zr * per);
    const int y = rem / sc.gdim[0], x = rem - y * sc.gdim[0];
    const long long node = sc.node_base + ((long long)(z0 + zr) * sc.gdim[1] + y) * sc.gdim[0] + x;
    float4* b0 = reinterpret_cast<float4*>(out ? out : const_cast<float*>(in));
    float4* b1 = b0 + total;
    float* bh = reinterpret_cast<float*>(b1 + total);
    if (out) {
      b0[i] = c.g.acc0[par][node];
      b1[i] = c.g.acc1[par][node];
      if (c.conduct) bh[i] = c.g.heat[par][node];
    } else if (node_active(c, sc, x, y, z0 + zr)) {
      const float4 p = c.g.acc0[par][node], q = b0[i];
      c.g.acc0[par][node] = make_float4(p.x + q.x, p.y + q.y, p.z + q.z, p.w + q.w);
      const float4 r = c.g.acc1[par][node], t = b1[i];
      c.g.acc1[par][node] = make_float4(r.x + t.x, r.y + t.y, r.z + t.z, r.w + t.w);
      if (c.conduct) c.g.heat[par][node] += bh[i];
    }
  }
}

void launch_halo_export(const Ctx& c, cudaStream_t st, int side, int planes, float* buf) {
  k_halo_copy<<<592, 256, 0, st>>>(c, side, planes, buf, nullptr);
}

void launch_halo_add(const Ctx& c, cudaStream_t st, int side, int planes, const float* buf) {
  k_halo_copy<<<592, 256, 0, st>>>(c, side, planes, nullptr, buf);
}

// Clears a pending scattered grid (acc[step_index & 1] over its active list) without using it.
__global__ void __launch_bounds__(256) k_grid_clear(Ctx c) {
  Ctrl* ct = c.ctrl;
  const int par = ct->step_index & 1;
  const unsigned count = ct->active_count[par];
  const int sub = threadIdx.x >> 6, lid = threadIdx.x & 63;
  for (unsigned ti = blockIdx.x * 4 + sub; ti < count; ti += gridDim.x * 4) {
    const unsigned tile = c.g.active[par][ti];
    const int s = c.nscenes == 1 ? 0 : find_scene_by_node_tile(c.scenes, c.nscenes, static_cast<int>(tile));
    const SceneDev& sc = c.scenes[s];
    const int lt = static_cast<int>(tile) - sc.node_tile_base;
    const int ntx = lt % sc.ntiles[0], nty = (lt / sc.ntiles[0]) % sc.ntiles[1], ntz = lt / (sc.ntiles[0] * sc.ntiles[1]);
    const int x = ntx * 4 + (lid & 3), y = nty * 4 + ((lid >> 2) & 3), z = ntz * 4 + (lid >> 4);
    const long long node = sc.node_base + ((long long)z * sc.gdim[1] + y) * sc.gdim[0] + x;
    c.g.acc0[par][node] = make_float4(0.f, 0.f, 0.f, 0.f);
    c.g.acc1[par][node] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (c.conduct) c.g.heat[par][node] = 0.f;
    if (lid == 0) c.g.tile_flag[tile] = 0u;
  }
}

void launch_grid_clear(const Ctx& c, cudaStream_t st, int grid_blocks) {
  k_grid_clear<<<grid_blocks, 256, 0, st>>>(c);
}

void launch_grid_update(const Ctx& c, cudaStream_t st, int grid_blocks) {
  k_grid_update<<<grid_blocks, 256, 0, st>>>(c);
}


// ---------------------------------------------------------------------------------------------
// FP64 ledger (src/simulation/mechanical-diagnostics.js:16-37, src/simulation/particle-health.js)

constexpr int kLedgerSums = 13;   // mass kin aff pot ela mom3 ang3
constexpr int kLedgerFields = 19; // + minJ maxJ maxEp maxVm nonfinite invalidJ

__device__ __forceinline__ double warp_sum(double x) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__global__ void __launch_bounds__(256) k_ledger(Ctx c, double* partials) {
  __shared__ double sh[8][kLedgerFields];
  double acc[kLedgerFields];
#pragma unroll
  for (int k = 0; k < kLedgerSums; ++k) acc[k] = 0.0;
  acc[13] = 1e300; acc[14] = -1e300; acc[15] = 0.0; acc[16] = 0.0; acc[17] = 0.0; acc[18] = 0.0;
  const long long cap = c.p.cap;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < c.n; i += (long long)gridDim.x * blockDim.x) {
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, i);
    const SceneDev& sc = c.scenes[s];
    const double Hs = sc.H;
    const double x[3] = {sc.origin[0] + c.p.qx[i] * (Hs / 4194304.0), sc.origin[1] + c.p.qy[i] * (Hs / 4194304.0),
                         sc.origin[2] + c.p.qz[i] * (Hs / 4194304.0)};
    const double v[3] = {c.p.vx[i], c.p.vy[i], c.p.vz[i]};
    float D[9], C[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      D[e] = c.p.D[e * cap + i];
      C[e] = c.p.C[e * cap + i];
    }
    const double m = c.p.m[i], V = c.p.V[i];
    const int mi = c.single_material ? sc.mat_base : c.p.mat[i];
    const MaterialDev mt = c.mats[mi];
    const double Dap = Hs * Hs / 4.0;
    acc[0] += m;
    acc[1] += 0.5 * m * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double c2 = 0.0;
#pragma unroll
    for (int e = 0; e < 9; ++e) c2 += (double)C[e] * C[e];
    acc[2] += 0.5 * m * Dap * c2;
    acc[3] -= m * (sc.gravity[0] * x[0] + sc.gravity[1] * x[1] + sc.gravity[2] * x[2]);
    const double P[3] = {m * v[0], m * v[1], m * v[2]};
    const double spin[3] = {(double)C[7] - C[5], (double)C[2] - C[6], (double)C[3] - C[1]};
    acc[5] += P[0]; acc[6] += P[1]; acc[7] += P[2];
    acc[8] += x[1] * P[2] - x[2] * P[1] + m * Dap * spin[0];
    acc[9] += x[2] * P[0] - x[0] * P[2] + m * Dap * spin[1];
    acc[10] += x[0] * P[1] - x[1] * P[0] + m * Dap * spin[2];
    // elastic energy density per reference volume by model
    const float Jm1 = det_minus_one(D);
    const double J = 1.0 + (double)Jm1;
    float Dc[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) Dc[e] = D[e];
    float aux = c.has_aux ? c.p.aux[i] : 0.f;
    const ConstitutiveOut co =
        constitutive_update_aux(mt, nullptr, Dc, 0.f, aux, c.has_thermal ? c.p.T[i] : 0.f, (float)(V / m), false);
    double W = 0.0;
    if (J > 0.0) {
      const Sym3 B = cauchy_green_minus_identity(D);
      if (mt.model == 1) {
        const double lj = log1p((double)Jm1);
        W = 0.5 * mt.mu * ((double)B.xx + B.yy + B.zz) - mt.mu * lj + 0.5 * mt.lam * lj * lj;
      } else {
        float beta[3], U[9];
        sym_eig3(B, beta, U);
        if (mt.model == 0 || mt.model == 2) {  // snow: fixed-corotated with its hardened moduli
          double s2 = 0.0;
          for (int kk = 0; kk < 3; ++kk) {
            const double sm1 = beta[kk] / (1.0 + sqrt(fmax(1.0 + beta[kk], 0.0)));
            s2 += sm1 * sm1;
          }
          W = (mt.model == 2 ? snow_hardening(aux) : 1.0) * (mt.mu * s2 + 0.5 * mt.lam * (double)Jm1 * Jm1);
        } else {
          double e2 = 0.0, tr = 0.0;
          for (int kk = 0; kk < 3; ++kk) {
            const double e = fmax(0.5 * log1p((double)beta[kk]), -13.815510558);
            e2 += e * e;
            tr += e;
          }
          W = mt.mu * e2 + 0.5 * mt.lam * tr * tr;
        }
      }
    }
    acc[4] += V * W;
    const double tvm = 0.5 * ((double)(co.tau.xx - co.tau.yy) * (co.tau.xx - co.tau.yy) +
                              (double)(co.tau.yy - co.tau.zz) * (co.tau.yy - co.tau.zz) +
                              (double)(co.tau.zz - co.tau.xx) * (co.tau.zz - co.tau.xx)) +
                       3.0 * ((double)co.tau.xy * co.tau.xy + (double)co.tau.xz * co.tau.xz + (double)co.tau.yz * co.tau.yz);
    // Cauchy von Mises; the pressure models divide by the total volume ratio J Jp (src/three/mpm.js:38)
    const double Jv = J * ((mt.model == 8 || mt.model == 9) ? 1.0 + (double)aux : 1.0);
    const double vm = sqrt(fmax(0.0, tvm)) / fmax(1e-6, Jv);
    bool finite = isfinite(m) && isfinite(v[0] + v[1] + v[2]) && isfinite(J) && isfinite(c2);
#pragma unroll
    for (int e = 0; e < 9; ++e) finite = finite && isfinite(D[e]);
    if (isfinite(J)) {
      acc[13] = fmin(acc[13], J);
      acc[14] = fmax(acc[14], J);
      if (J <= 0.0) acc[18] += 1.0;
    }
    if (c.has_plastic) acc[15] = fmax(acc[15], (double)c.p.ep[i]);
    if (isfinite(vm)) acc[16] = fmax(acc[16], vm);
    if (!finite) acc[17] += 1.0;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kLedgerSums; ++k) acc[k] = warp_sum(acc[k]);
  for (int o = 16; o > 0; o >>= 1) {
    acc[13] = fmin(acc[13], __shfl_xor_sync(0xffffffffu, acc[13], o));
    acc[14] = fmax(acc[14], __shfl_xor_sync(0xffffffffu, acc[14], o));
    acc[15] = fmax(acc[15], __shfl_xor_sync(0xffffffffu, acc[15], o));
    acc[16] = fmax(acc[16], __shfl_xor_sync(0xffffffffu, acc[16], o));
  }
  acc[17] = warp_sum(acc[17]);
  acc[18] = warp_sum(acc[18]);
  if (lane == 0)
    for (int k = 0; k < kLedgerFields; ++k) sh[wid][k] = acc[k];
  __syncthreads();
  if (threadIdx.x < kLedgerFields) {
    const int k = threadIdx.x;
    double r = sh[0][k];
    for (int w = 1; w < 8; ++w) {
      const double y = sh[w][k];
      if (k == 13) r = fmin(r, y);
      else if (k >= 14 && k <= 16) r = fmax(r, y);
      else r += y;
    }
    partials[blockIdx.x * kLedgerFields + k] = r;
  }
}

// Deterministic final reduction of the per-block partials (fixed order).
__global__ void k_ledger_final(const double* partials, int blocks, double* out) {
  const int k = threadIdx.x;
  if (k >= kLedgerFields) return;
  double r = (k == 13) ? 1e300 : (k >= 14 && k <= 16) ? -1e300 : 0.0;
  if (k == 15 || k == 16) r = 0.0;
  for (int b = 0; b < blocks; ++b) {
    const double y = partials[b * kLedgerFields + k];
    if (k == 13) r = fmin(r, y);
    else if (k >= 14 && k <= 16) r = fmax(r, y);
    else r += y;
  }
  out[k] = r;
}

void launch_ledger(const Ctx& c, cudaStream_t st, double* partials, int blocks, double* out) {
  k_ledger<<<blocks, 256, 0, st>>>(c, partials);
  k_ledger_final<<<1, 32, 0, st>>>(partials, blocks, out);
}

// Grid after P2G of one scene in the reference's node order: mass and p + dt (f + m g).
__global__ void k_grid_debug(Ctx c, int scene, float dt, double* mass, double* mom) {
  const SceneDev& sc = c.scenes[scene];
  const int nx = sc.dims[0], ny = sc.dims[1], nz = sc.dims[2];
  const long long total = (long long)nx * ny * nz;
  const int par = c.ctrl->step_index & 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = static_cast<int>(i % nx), y = static_cast<int>((i / nx) % ny), z = static_cast<int>(i / ((long long)nx * ny));
    const long long node = sc.node_base + ((long long)z * sc.gdim[1] + y) * sc.gdim[0] + x;
    const float4 a0 = c.g.acc0[par][node], a1 = c.g.acc1[par][node];
    mass[i] = a0.x;
    mom[i * 3 + 0] = (double)a0.y + (double)dt * ((double)a1.x + (double)a0.x * sc.gravity[0]);
    mom[i * 3 + 1] = (double)a0.z + (double)dt * ((double)a1.y + (double)a0.x * sc.gravity[1]);
    mom[i * 3 + 2] = (double)a0.w + (double)dt * ((double)a1.z + (double)a0.x * sc.gravity[2]);
  }
}

void launch_grid_debug(const Ctx& c, cudaStream_t st, int scene, float dt, double* mass, double* mom) {
  k_grid_debug<<<1024, 256, 0, st>>>(c, scene, dt, mass, mom);
}

// ---------------------------------------------------------------------------------------------
// host <-> device conversion (staging buffers hold the caller's f64 or f32 arrays)

// Host arrays (staged on the device) into the SoA state. A full upload sets the home order to the
// caller's order (id = i); with by_id the caller's particle id[i] is read into home slot i.
template <typename Tsrc>
__global__ void k_upload(Ctx c, long long n, const Tsrc* const* src, const int* material,
                         const unsigned char* pinned, unsigned fields, int by_id, const unsigned char* melted) {
  const long long cap = c.p.cap;
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < n; h += (long long)gridDim.x * blockDim.x) {
    const long long i = by_id ? (long long)c.p.id[h] : h;
    if (!by_id) c.p.id[h] = static_cast<unsigned>(h);
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, h);
    const SceneDev& sc = c.scenes[s];
    if (fields & kFieldPos) {
      unsigned* qs[3] = {c.p.qx, c.p.qy, c.p.qz};
      for (int a = 0; a < 3; ++a) {
        const double q = rint(((double)src[a][i] - sc.origin[a]) / (double)sc.H * 4194304.0);
        const double hi = (double)(((long long)sc.dims[a] - 1) << kFracBits);
        qs[a][h] = static_cast<unsigned>(fmin(fmax(q, 0.0), hi));
      }
    }
    if (fields & kFieldVel) {
      c.p.vx[h] = src[3] ? (float)src[3][i] : 0.f;
      c.p.vy[h] = src[4] ? (float)src[4][i] : 0.f;
      c.p.vz[h] = src[5] ? (float)src[5][i] : 0.f;
    }
    if (fields & kFieldMass) c.p.m[h] = (float)src[6][i];
    if (fields & kFieldVolume) c.p.V[h] = (float)src[7][i];
    if (fields & kFieldTemp) {
      // temperature, or the decode of the enthalpy (src/three/phase-change.js:12-18); the molten
      // flag is the hint on a latent plateau, else follows from T > melting point (phaseEnthalpy)
      const int mi = material ? sc.mat_base + material[i] : sc.mat_base;
      const MaterialExt& xt = c.mats_ext[mi];
      const double cp = c.mats[mi].cp;
      double T = src[8] ? (double)src[8][i] : 0.0;
      float f = 0.f;
      unsigned char mol = melted ? melted[i] : 0;
      if (src[14] && xt.latent > 0.f) {
        const double hh = (double)src[14][i], start = cp * xt.melting_point, end = start + xt.latent;
        if (hh <= start) { T = hh / cp; f = 0.f; mol = 0; }
        else if (hh >= end) { T = (hh - xt.latent) / cp; f = 1.f; mol = 1; }
        else { T = xt.melting_point; f = (float)((hh - start) / xt.latent); }
      } else if (src[14] && cp > 0.0) {
        T = (double)src[14][i] / cp;
        mol = 0;
      } else if (xt.latent > 0.f) {
        mol = T > xt.melting_point ? 1 : 0;
        f = mol ? 1.f : 0.f;
      } else {
        mol = 0;
      }
      c.p.T[h] = (float)T;
      c.p.latent[h] = f;
      c.p.melted[h] = mol;
    }
    if (fields & kFieldPlastic) c.p.ep[h] = src[9] ? (float)src[9][i] : 0.f;
    if (fields & kFieldAux) {
      // aux = Jp - 1 (models 2, 8, 9) or the dilation (model 3)
      const int model = c.mats[material ? sc.mat_base + material[i] : sc.mat_base].model;
      float a = 0.f;
      if ((model == 2 || model == 8 || model == 9) && src[12]) a = (float)((double)src[12][i] - 1.0);
      if (model == 3 && src[13]) a = (float)src[13][i];
      c.p.aux[h] = a;
    }
    if (fields & kFieldF)
      for (int e = 0; e < 9; ++e)
        c.p.D[e * cap + h] = src[10] ? (float)((double)src[10][i * 9 + e] - ((e % 4 == 0) ? 1.0 : 0.0)) : 0.f;
    if (fields & kFieldC)
      for (int e = 0; e < 9; ++e) c.p.C[e * cap + h] = src[11] ? (float)src[11][i * 9 + e] : 0.f;
    if (fields & kFieldMass) {
      c.p.mat[h] = material ? static_cast<unsigned short>(sc.mat_base + material[i])
                            : static_cast<unsigned short>(sc.mat_base);
      if (c.p.pinned) c.p.pinned[h] = pinned ? pinned[i] : 0;
    }
  }
}

void launch_upload_convert(const Ctx& c, cudaStream_t st, long long n, int dtype, const void* const* src,
                           const int* material, const unsigned char* pinned, unsigned fields, bool by_id,
                           const unsigned char* melted) {
  if (n <= 0) return;
  const int blocks = static_cast<int>((n + 255) / 256 < 65536 ? (n + 255) / 256 : 65536);
  if (dtype == 0)
    k_upload<double><<<blocks, 256, 0, st>>>(c, n, reinterpret_cast<const double* const*>(src), material, pinned, fields,
                                             by_id ? 1 : 0, melted);
  else
    k_upload<float><<<blocks, 256, 0, st>>>(c, n, reinterpret_cast<const float* const*>(src), material, pinned, fields,
                                            by_id ? 1 : 0, melted);
}

// Rewrites the state in sort order: dst[i] = current[perm[i]] for every field, then perm = identity,
// so each tile's particles are contiguous in every array.
__global__ void k_permute(Ctx c, Particles d) {
  const Particles& s = c.p;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < c.n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned h = s.perm[i];
    d.qx[i] = s.qx[h]; d.qy[i] = s.qy[h]; d.qz[i] = s.qz[h];
    d.vx[i] = s.vx[h]; d.vy[i] = s.vy[h]; d.vz[i] = s.vz[h];
#pragma unroll
    for (int e = 0; e < 9; ++e) {
      d.Cc[e][i] = s.Cc[e][h];
      d.Dc[e][i] = s.Dc[e][h];
    }
    d.m[i] = s.m[h]; d.V[i] = s.V[h]; d.ep[i] = s.ep[h]; d.T[i] = s.T[h]; d.aux[i] = s.aux[h];
    d.latent[i] = s.latent[h]; d.melted[i] = s.melted[h];
    d.mat[i] = s.mat[h]; d.pinned[i] = s.pinned[h]; d.id[i] = s.id[h];
    s.perm[i] = static_cast<unsigned>(i);
  }
}

// Before a permutation: orders each tile's perm range by the particle's stencil base cell within
// the tile (64 cells; counting sort in shared memory, one CTA per tile of the current work list),
// so after the permutation the particles of one cell sit in consecutive home slots and a warp of
// consecutive particles touches few cells. Tiles above kCellSortMax particles keep their order.
constexpr int kCellSortMax = 4096;

__global__ void __launch_bounds__(256) k_cell_order(Ctx c) {
  __shared__ unsigned ids[kCellSortMax];
  __shared__ unsigned char cell[kCellSortMax];
  __shared__ int cursor[64];
  const unsigned list = c.ctrl->step_index & 1u;
  const unsigned nwork = min(c.ctrl->work_count[list], static_cast<unsigned>(c.total_tiles));
  for (unsigned w = blockIdx.x; w < nwork; w += gridDim.x) {
    const uint4 it = c.s.work[list][w];  // (tile, start, count, scene)
    if (it.z > static_cast<unsigned>(kCellSortMax) || it.y + it.z > static_cast<unsigned long long>(c.n)) continue;
    const SceneDev& sc = c.scenes[it.w];
    if (threadIdx.x < 64) cursor[threadIdx.x] = 0;
    __syncthreads();
    for (unsigned j = threadIdx.x; j < it.z; j += blockDim.x) {
      const unsigned h = c.p.perm[it.y + j];
      int b0, b1, b2;
      float t;
      stencil_axis(c.p.qx[h], sc.dims[0], b0, t);
      stencil_axis(c.p.qy[h], sc.dims[1], b1, t);
      stencil_axis(c.p.qz[h], sc.dims[2], b2, t);
      const int local = ((b2 & 3) * 4 + (b1 & 3)) * 4 + (b0 & 3);
      ids[j] = h;
      cell[j] = static_cast<unsigned char>(local);
      atomicAdd(&cursor[local], 1);
    }
    __syncthreads();
    if (threadIdx.x < 32) {  // exclusive scan of the 64 cell counts by one warp (two per lane)
      const int a0 = cursor[2 * threadIdx.x], a1 = cursor[2 * threadIdx.x + 1];
      int inc = a0 + a1;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (threadIdx.x >= o) inc += y;
      }
      const int ex = inc - a0 - a1;
      cursor[2 * threadIdx.x] = ex;
      cursor[2 * threadIdx.x + 1] = ex + a0;
    }
    __syncthreads();
    for (unsigned j = threadIdx.x; j < it.z; j += blockDim.x) {
      const int pos = atomicAdd(&cursor[cell[j]], 1);
      c.p.perm[it.y + pos] = ids[j];
    }
    __syncthreads();
  }
}

void launch_permute(const Ctx& c, const Particles& dst, cudaStream_t st) {
  if (c.n <= 0) return;
  const int tiles = c.total_tiles < 4096 ? c.total_tiles : 4096;
  if (tiles > 0) k_cell_order<<<tiles, 256, 0, st>>>(c);
  const long long blocks = (c.n + 255) / 256 < 65536 ? (c.n + 255) / 256 : 65536;
  k_permute<<<static_cast<unsigned>(blocks), 256, 0, st>>>(c, dst);
}

// Home slots of the caller's particle indices a and b (slots[0], slots[1]; -1 when absent).
__global__ void k_find_ids(Ctx c, unsigned a, unsigned b, long long* slots) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < c.n; i += (long long)gridDim.x * blockDim.x) {
    const unsigned id = c.p.id[i];
    if (id == a) slots[0] = i;
    if (id == b) slots[1] = i;
  }
}

__device__ void copy_slot(const Particles& p, long long dst, long long src) {
  p.qx[dst] = p.qx[src]; p.qy[dst] = p.qy[src]; p.qz[dst] = p.qz[src];
  p.vx[dst] = p.vx[src]; p.vy[dst] = p.vy[src]; p.vz[dst] = p.vz[src];
  for (int e = 0; e < 9; ++e) {
    p.Cc[e][dst] = p.Cc[e][src];
    p.Dc[e][dst] = p.Dc[e][src];
  }
  p.m[dst] = p.m[src]; p.V[dst] = p.V[src]; p.ep[dst] = p.ep[src]; p.T[dst] = p.T[src]; p.aux[dst] = p.aux[src];
  p.latent[dst] = p.latent[src]; p.melted[dst] = p.melted[src];
  p.mat[dst] = p.mat[src]; p.pinned[dst] = p.pinned[src]; p.id[dst] = p.id[src];
}

// op 0: MPM3.resetParticle of the particle in slots[0] (src/three/mpm.js:21).
// op 1: MPM3.remove(p, last) (src/three/mpm.js:22-25): the particle in slots[1] (caller index
// last) takes caller index p, the particle in slots[0] (caller index p) is dropped, and home slot
// n - 1 moves into the freed slot so the live slots stay [0, n - 1). The host has checked that
// both slots exist.
__global__ void k_edit_particle(Ctx c, int op, unsigned new_id, const long long* slots) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const long long sp = slots[0], sl = slots[1];
  if (sp < 0 || sp >= c.n || (op == 1 && (sl < 0 || sl >= c.n))) return;
  if (op == 0) {
    for (int e = 0; e < 9; ++e) {
      c.p.Cc[e][sp] = 0.f;
      c.p.Dc[e][sp] = 0.f;
    }
    c.p.ep[sp] = 0.f;
    c.p.aux[sp] = 0.f;  // Jp = 1, dilation = 0
    return;
  }
  c.p.id[sl] = new_id;
  const long long last = c.n - 1;
  if (sp != last) copy_slot(c.p, sp, last);
}

void launch_find_ids(const Ctx& c, cudaStream_t st, unsigned a, unsigned b, long long* slots) {
  cudaMemsetAsync(slots, 0xff, 2 * sizeof(long long), st);
  const long long blocks = (c.n + 255) / 256 < 4096 ? (c.n + 255) / 256 : 4096;
  if (blocks > 0) k_find_ids<<<static_cast<unsigned>(blocks), 256, 0, st>>>(c, a, b, slots);
}

void launch_edit_particle(const Ctx& c, cudaStream_t st, int op, unsigned a, const long long* slots) {
  k_edit_particle<<<1, 32, 0, st>>>(c, op, a, slots);
}

template <typename Tdst>
__global__ void k_download(Ctx c, long long n, Tdst* const* dst, unsigned fields) {
  const long long cap = c.p.cap;
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < n; h += (long long)gridDim.x * blockDim.x) {
    const long long i = c.p.id[h];  // caller's index of home slot h
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, h);
    const SceneDev& sc = c.scenes[s];
    if (fields & kFieldPos) {
      const unsigned q[3] = {c.p.qx[h], c.p.qy[h], c.p.qz[h]};
      for (int a = 0; a < 3; ++a) dst[a][i] = (Tdst)(sc.origin[a] + (double)q[a] * ((double)sc.H / 4194304.0));
    }
    if (fields & kFieldVel) {
      dst[3][i] = (Tdst)c.p.vx[h];
      dst[4][i] = (Tdst)c.p.vy[h];
      dst[5][i] = (Tdst)c.p.vz[h];
    }
    if (fields & kFieldMass) dst[6][i] = (Tdst)c.p.m[h];
    if (fields & kFieldVolume) dst[7][i] = (Tdst)c.p.V[h];
    if (fields & kFieldTemp) {
      if (dst[8]) dst[8][i] = (Tdst)c.p.T[h];
      if (dst[14]) {  // h = cp T (+ the molten fraction of the latent heat)
        const int mi = c.single_material ? sc.mat_base : c.p.mat[h];
        dst[14][i] = (Tdst)((double)c.mats[mi].cp * c.p.T[h] + (double)c.p.latent[h] * c.mats_ext[mi].latent);
      }
    }
    if (fields & kFieldPlastic) dst[9][i] = (Tdst)c.p.ep[h];
    if (fields & kFieldAux) {
      const int model = c.mats[c.single_material ? sc.mat_base : c.p.mat[h]].model;
      const double a = c.p.aux[h];
      if (dst[12]) dst[12][i] = (Tdst)((model == 2 || model == 8 || model == 9) ? 1.0 + a : 1.0);
      if (dst[13]) dst[13][i] = (Tdst)(model == 3 ? a : 0.0);
    }
    for (int e = 0; e < 9; ++e) {
      const double ident = (e % 4 == 0) ? 1.0 : 0.0;
      if (fields & kFieldF) dst[10][i * 9 + e] = (Tdst)((double)c.p.D[e * cap + h] + ident);
      if (fields & kFieldC) dst[11][i * 9 + e] = (Tdst)c.p.C[e * cap + h];
    }
  }
}

__global__ void k_download_melted(Ctx c, long long n, unsigned char* out) {
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < n; h += (long long)gridDim.x * blockDim.x)
    out[c.p.id[h]] = c.p.melted[h];
}

void launch_download_melted(const Ctx& c, cudaStream_t st, long long n, unsigned char* out) {
  if (n <= 0) return;
  const int blocks = static_cast<int>((n + 255) / 256 < 65536 ? (n + 255) / 256 : 65536);
  k_download_melted<<<blocks, 256, 0, st>>>(c, n, out);
}

void launch_download_convert(const Ctx& c, cudaStream_t st, long long n, int dtype, void* const* dst, unsigned fields) {
  if (n <= 0) return;
  const int blocks = static_cast<int>((n + 255) / 256 < 65536 ? (n + 255) / 256 : 65536);
  if (dtype == 0)
    k_download<double><<<blocks, 256, 0, st>>>(c, n, reinterpret_cast<double* const*>(dst), fields);
  else
    k_download<float><<<blocks, 256, 0, st>>>(c, n, reinterpret_cast<float* const*>(dst), fields);
}

// ---------------------------------------------------------------------------------------------
// Frame packing for a viewer (gpu/solver.py:985-1035): one deterministic sample per block of
// `stride` caller indices, chosen by the reference's integer hash so previews show no lattice
// stripes, as 8 floats (x, y, z, material, T, pinned, von Mises stress, plastic strain), plus the
// frame reductions the ledger does not carry. stats: [0] sum m cp T (FP64), [1] ordered-key
// min T, [2] ordered-key max T (as doubles holding the keys), counts[256]: particles per material.

__device__ __forceinline__ unsigned preview_pick(unsigned row, unsigned span) {
  unsigned h = row * 747796405u + 2891336453u;
  h = ((h >> ((h >> 28) + 4u)) ^ h) * 277803737u;
  h = (h >> 22) ^ h;
  return h % span;
}

__device__ __forceinline__ unsigned ordered_key(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_pack_frame(Ctx c, long long stride, float* data, double* energy, unsigned* tkey, unsigned* counts) {
  double e_acc = 0.0;
  unsigned tmin = 0xffffffffu, tmax = 0u;
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < c.n; h += (long long)gridDim.x * blockDim.x) {
    const long long id = c.p.id[h];
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, h);
    const SceneDev& sc = c.scenes[s];
    const int mi = c.single_material ? sc.mat_base : c.p.mat[h];
    const MaterialDev& mt = c.mats[mi];
    const float T = c.has_thermal ? c.p.T[h] : 0.f;
    const float m = c.p.m[h];
    e_acc += (double)m * mt.cp * T;
    tmin = min(tmin, ordered_key(T));
    tmax = max(tmax, ordered_key(T));
    {  // one atomic per distinct material in the warp
      const unsigned peers = __match_any_sync(__activemask(), mi);
      if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&counts[mi], __popc(peers));
    }
    const long long row = id / stride;
    const long long span = min(stride, c.n - row * stride);
    if ((id % stride) != (long long)preview_pick(static_cast<unsigned>(row), static_cast<unsigned>(span))) continue;
    float D[9];
    for (int e = 0; e < 9; ++e) D[e] = c.p.D[e * c.p.cap + h];
    const float Jm1 = det_minus_one(D);
    float aux = c.has_aux ? c.p.aux[h] : 0.f;
    const ConstitutiveOut co = constitutive_update_aux(mt, nullptr, D, 0.f, aux, T, c.p.V[h] / m, false);
    const float dxy = co.tau.xx - co.tau.yy, dyz = co.tau.yy - co.tau.zz, dzx = co.tau.zz - co.tau.xx;
    const float vm = sqrtf(fmaxf(0.f, 0.5f * (dxy * dxy + dyz * dyz + dzx * dzx) +
                                          3.f * (co.tau.xy * co.tau.xy + co.tau.xz * co.tau.xz + co.tau.yz * co.tau.yz))) /
                     fmaxf(1e-6f, (1.f + Jm1) * ((mt.model == 8 || mt.model == 9) ? 1.f + aux : 1.f));
    float* r = data + row * 8;
    const double Hs = sc.H;
    r[0] = (float)(sc.origin[0] + c.p.qx[h] * (Hs / 4194304.0));
    r[1] = (float)(sc.origin[1] + c.p.qy[h] * (Hs / 4194304.0));
    r[2] = (float)(sc.origin[2] + c.p.qz[h] * (Hs / 4194304.0));
    r[3] = (float)mi;
    r[4] = T;
    r[5] = c.has_pinned ? (float)c.p.pinned[h] : 0.f;
    r[6] = vm;
    r[7] = c.has_plastic ? c.p.ep[h] : 0.f;
  }
  const double es = warp_sum_d(e_acc);
  const unsigned mn = __reduce_min_sync(0xffffffffu, tmin), mx = __reduce_max_sync(0xffffffffu, tmax);
  if ((threadIdx.x & 31) == 0) {
    if (es != 0.0) atomicAdd(energy, es);
    atomicMin(&tkey[0], mn);
    atomicMax(&tkey[1], mx);
  }
}

void launch_pack_frame(const Ctx& c, cudaStream_t st, long long stride, float* data, double* energy, unsigned* tkey,
                       unsigned* counts) {
  const long long blocks = (c.n + 255) / 256 < 4096 ? (c.n + 255) / 256 : 4096;
  if (blocks > 0) k_pack_frame<<<static_cast<unsigned>(blocks), 256, 0, st>>>(c, stride, data, energy, tkey, counts);
}

// ---------------------------------------------------------------------------------------------
// stateless constitutive batch: projectPlastic + stress (src/three/constitutive.js:52-86)

__global__ void k_return_map(MaterialDev mt, long long n, const double* F_in, const double* ep, const double* T,
                             float dt, double* F_out, double* dep, double* tau) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float D[9];
    for (int e = 0; e < 9; ++e) D[e] = (float)(F_in[i * 9 + e] - ((e % 4 == 0) ? 1.0 : 0.0));
    const float epi = ep ? (float)ep[i] : 0.f, Ti = T ? (float)T[i] : 0.f;
    const ConstitutiveOut co = constitutive_update(mt, D, epi, Ti, 1.f, true, dt);
    for (int e = 0; e < 9; ++e) F_out[i * 9 + e] = (double)D[e] + ((e % 4 == 0) ? 1.0 : 0.0);
    dep[i] = co.dep;
    const float t9[9] = {co.tau.xx, co.tau.xy, co.tau.xz, co.tau.xy, co.tau.yy, co.tau.yz, co.tau.xz, co.tau.yz, co.tau.zz};
    for (int e = 0; e < 9; ++e) tau[i * 9 + e] = t9[e];
  }
}

void launch_return_map_batch(const MaterialDev& m, long long n, const double* F_in, const double* ep, const double* T,
                             float dt, double* F_out, double* dep, double* tau, cudaStream_t st) {
  const int blocks = static_cast<int>((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
  if (blocks > 0) k_return_map<<<blocks, 256, 0, st>>>(m, n, F_in, ep, T, dt, F_out, dep, tau);
}

}  // namespace mpm
