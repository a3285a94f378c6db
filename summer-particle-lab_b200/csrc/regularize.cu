// Solid position regularisation on the device (src/three/solid-sampling.js:5-42, regularizeSolids;
// the reference's GPU twin is gpu/solver.py:565-648).
//
// Per pass:
//   k_reg_count    thread per particle: neighbour cell (cells as large as the largest target, two
//                  spacings, so every pair closer than its target lies in the 27 surrounding
//                  cells), target spacing from V J Jp, cell population
//   scan           exclusive prefix sum of the populations (k_scan_blocks / k_scan_top / k_scan_add)
//   k_reg_scatter  particle slots grouped by cell, with a packed copy of what the pair test reads
//                  (position, target, inverse mass, index, material) in cell order, so neighbour
//                  candidates are read as contiguous runs
//   k_reg_pairs    thread per particle in cell order: its own shift, gathered over the 27 cells.
//                  The reference visits each pair once (i < j) and adds +shift to i and -shift to j; the pair
//                  term is antisymmetric, so gathering every neighbour from each side gives the
//                  same sums without atomics. The largest shift of each scene over its budget.
//   k_reg_apply    x += shift / max(1, largest / budget) for unpinned particles, clamped to the box
// HBM traffic per particle: about 110 B (position, D, V, m, aux, id reads; the cell, target, shift
// and packed scratch) plus the neighbour reads, contiguous runs of the packed copy that L1/L2 serve.
#include "mpm_internal.h"
#include "regularize.h"

namespace mpm {

namespace {

__device__ __forceinline__ void position(const Particles& p, long long h, const SceneDev& sc, float x[3]) {
  // metres from the scene's grid origin (exact integer cell part, FP32 fraction)
  const unsigned q[3] = {p.qx[h], p.qy[h], p.qz[h]};
  for (int a = 0; a < 3; ++a) x[a] = static_cast<float>(q[a]) * kInvFixedOne * sc.H;
}

__global__ void k_reg_count(Ctx c, RegDev r, unsigned* cell_of, float* target, float* inv_mass, unsigned* count) {
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < c.n; h += (long long)gridDim.x * blockDim.x) {
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, h);
    const SceneDev& sc = c.scenes[s];
    const RegScene& rs = r.scenes[s];
    float x[3];
    position(c.p, h, sc, x);
    int cc[3];
    for (int a = 0; a < 3; ++a) cc[a] = min(rs.nc[a] - 1, max(0, static_cast<int>(floorf(x[a] * r.inv_hc))));
    const unsigned cell = static_cast<unsigned>(rs.cell_base + ((long long)cc[2] * rs.nc[1] + cc[1]) * rs.nc[0] + cc[0]);
    cell_of[h] = cell;
    atomicAdd(&count[cell], 1u);
    // spacing 2.8 cbrt(clamp(V J Jp, 1/64, 8)) in the reference's units (solid-sampling.js:5-8)
    const int mi = c.single_material ? sc.mat_base : c.p.mat[h];
    const int model = c.mats[mi].model;
    float D[9];
    for (int e = 0; e < 9; ++e) D[e] = c.p.Dc[e][h];
    const float J = 1.f + det_minus_one(D);
    const float jp = (c.has_aux && (model == 2 || model == 8 || model == 9)) ? 1.f + c.p.aux[h] : 1.f;
    const float vol = fminf(8.f, fmaxf(0.015625f, c.p.V[h] * J * jp * r.inv_volume_unit));
    target[h] = r.spacing * cbrtf(vol);
    inv_mass[h] = (c.has_pinned && c.p.pinned[h]) ? 0.f : 1.f / c.p.m[h];
  }
}

__global__ void k_reg_scatter(Ctx c, const unsigned* cell_of, const unsigned* start, unsigned* cursor,
                              const float* target, const float* inv_mass, unsigned* sorted, uint4* pos_sorted,
                              uint2* inv_sorted, unsigned short* mat_sorted) {
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < c.n; h += (long long)gridDim.x * blockDim.x) {
    const unsigned cell = cell_of[h];
    const unsigned k = start[cell] + atomicAdd(&cursor[cell], 1u);
    sorted[k] = static_cast<unsigned>(h);
    pos_sorted[k] = make_uint4(c.p.qx[h], c.p.qy[h], c.p.qz[h], __float_as_uint(target[h]));
    inv_sorted[k] = make_uint2(__float_as_uint(inv_mass[h]), c.p.id[h]);
    if (!c.single_material) mat_sorted[k] = c.p.mat[h];
  }
}

__device__ __forceinline__ float scene_dt(const RegDev& r, int s) { return r.dt_scene ? r.dt_scene[s] : r.dt; }

__global__ void k_reg_pairs(Ctx c, RegDev r, const unsigned* cell_of, const unsigned* start, const unsigned* count,
                            const unsigned* sorted, const uint4* pos_sorted, const uint2* inv_sorted,
                            const unsigned short* mat_sorted, float4* shift, unsigned* largest) {
  for (long long ks = blockIdx.x * (long long)blockDim.x + threadIdx.x; ks < c.n; ks += (long long)gridDim.x * blockDim.x) {
    const unsigned i = sorted[ks];  // home slot
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, i);
    const SceneDev& sc = c.scenes[s];
    const RegScene& rs = r.scenes[s];
    const float dt = scene_dt(r, s);
    const float gain = -expm1f(-r.rate * dt);
    const uint4 pi = pos_sorted[ks];
    const uint2 bi = inv_sorted[ks];
    const unsigned qi[3] = {pi.x, pi.y, pi.z};
    const float ti = __uint_as_float(pi.w), inv_i = __uint_as_float(bi.x);
    const unsigned id_i = bi.y;
    const int mat_i = c.single_material ? 0 : mat_sorted[ks];
    const float to_m = sc.H * kInvFixedOne;
    const long long local = (long long)cell_of[i] - rs.cell_base;
    const int cx = static_cast<int>(local % rs.nc[0]), cy = static_cast<int>((local / rs.nc[0]) % rs.nc[1]),
              cz = static_cast<int>(local / ((long long)rs.nc[0] * rs.nc[1]));
    float acc[3] = {0.f, 0.f, 0.f};
    if (inv_i > 0.f) {  // a pinned particle's own shift is never applied
      for (int z = max(0, cz - 1); z <= min(rs.nc[2] - 1, cz + 1); ++z)
        for (int y = max(0, cy - 1); y <= min(rs.nc[1] - 1, cy + 1); ++y)
          for (int x = max(0, cx - 1); x <= min(rs.nc[0] - 1, cx + 1); ++x) {
            const long long cell = rs.cell_base + ((long long)z * rs.nc[1] + y) * rs.nc[0] + x;
            const unsigned b = start[cell], e = b + count[cell];
            for (unsigned k = b; k < e; ++k) {
              if (k == ks) continue;
              if (!c.single_material && mat_sorted[k] != mat_i) continue;  // one part
              const uint4 pj = pos_sorted[k];
              // exact fixed-point differences, then metres
              float d[3] = {static_cast<float>(static_cast<int>(qi[0] - pj.x)) * to_m,
                            static_cast<float>(static_cast<int>(qi[1] - pj.y)) * to_m,
                            static_cast<float>(static_cast<int>(qi[2] - pj.z)) * to_m};
              float rr = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
              const float t = 0.5f * (ti + __uint_as_float(pj.w));
              if (!(rr < t)) continue;
              const uint2 bj = inv_sorted[k];
              const float total = inv_i + __uint_as_float(bj.x);
              float q;
              if (rr < r.eps) {
                // the reference's hashed direction of the pair (lower index first), +/- by side
                const unsigned id_j = bj.y;
                const unsigned lo = min(id_i, id_j), hi = max(id_i, id_j);
                const unsigned hsh = (lo + 1u) * 73856093u ^ (hi + 1u) * 19349663u;
                const float sign = id_i < id_j ? 1.f : -1.f;
                d[0] = sign * (static_cast<float>(hsh & 1023u) / 511.5f - 1.f);
                d[1] = sign * (static_cast<float>((hsh >> 10) & 1023u) / 511.5f - 1.f);
                d[2] = sign * (static_cast<float>((hsh >> 20) & 1023u) / 511.5f - 1.f);
                rr = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                q = t * gain / (rr * total);
              } else {
                q = (t - rr) * gain / (rr * total);
              }
              acc[0] += d[0] * q;
              acc[1] += d[1] * q;
              acc[2] += d[2] * q;
            }
          }
    }
    const float sx = acc[0] * inv_i, sy = acc[1] * inv_i, sz = acc[2] * inv_i;
    shift[i] = make_float4(sx, sy, sz, 0.f);
    // the reference takes the largest shift over every solid, pinned ones included (a pinned
    // particle's is zero here since its inverse mass is zero)
    const float over = sqrtf(sx * sx + sy * sy + sz * sz) / (r.max_speed * dt);
    if (over > 1.f) atomicMax(&largest[s], __float_as_uint(over));
  }
}

__global__ void k_reg_apply(Ctx c, RegDev r, const float4* shift, const unsigned* largest) {
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < c.n; h += (long long)gridDim.x * blockDim.x) {
    if (c.has_pinned && c.p.pinned[h]) continue;
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, h);
    const SceneDev& sc = c.scenes[s];
    const float scale = fmaxf(1.f, __uint_as_float(largest[s]));
    const float4 d = shift[h];
    const float k = sc.invH * kFixedOne / scale;
    unsigned* qs[3] = {c.p.qx, c.p.qy, c.p.qz};
    const float dd[3] = {d.x, d.y, d.z};
    for (int a = 0; a < 3; ++a) {
      long long q = static_cast<long long>(qs[a][h]) + __float2ll_rn(dd[a] * k);
      const long long lo = sc.clamp ? (long long)sc.qlo[a] : 0;
      const long long hi = sc.clamp ? (long long)sc.qhi[a] : ((long long)sc.dims[a] - 1) << kFracBits;
      qs[a][h] = static_cast<unsigned>(q < lo ? lo : (q > hi ? hi : q));
    }
  }
}

// Exclusive scan of n unsigned counts into out, in three launches (4096 per block).
constexpr int kScanThreads = 1024, kScanItems = 4;
constexpr int kScanSpan = kScanThreads * kScanItems;

__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned* warp_sums, unsigned* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    warp_sums[lane] = s;  // inclusive over warps
  }
  __syncthreads();
  const unsigned before = (w > 0 ? warp_sums[w - 1] : 0u) + x - v;
  if (total) *total = warp_sums[(blockDim.x >> 5) - 1];
  return before;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(const unsigned* in, long long n, unsigned* out,
                                                             unsigned* block_sums) {
  __shared__ unsigned ws[32];
  __shared__ unsigned tot;
  const long long base = (long long)blockIdx.x * kScanSpan + (long long)threadIdx.x * kScanItems;
  unsigned v[kScanItems], sum = 0;
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0u;
    sum += v[k];
  }
  unsigned t = 0;
  unsigned run = block_exclusive_scan(sum, ws, threadIdx.x == 0 ? &t : nullptr);
  if (threadIdx.x == 0) tot = t;
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// One block scans the block sums in place (up to kScanSpan of them), chunk by chunk.
__global__ void __launch_bounds__(kScanThreads) k_scan_top(unsigned* block_sums, int nb) {
  __shared__ unsigned ws[32];
  unsigned carry = 0;
  for (int base = 0; base < nb; base += kScanSpan) {
    const int b = base + threadIdx.x * kScanItems;
    unsigned v[kScanItems], sum = 0;
    for (int k = 0; k < kScanItems; ++k) {
      v[k] = b + k < nb ? block_sums[b + k] : 0u;
      sum += v[k];
    }
    __shared__ unsigned tot;
    unsigned t = 0;
    unsigned run = carry + block_exclusive_scan(sum, ws, threadIdx.x == 0 ? &t : nullptr);
    if (threadIdx.x == 0) tot = t;
    for (int k = 0; k < kScanItems; ++k) {
      if (b + k < nb) block_sums[b + k] = run;
      run += v[k];
    }
    __syncthreads();
    carry += tot;
    __syncthreads();
  }
}

__global__ void k_scan_add(unsigned* out, long long n, const unsigned* block_sums) {
  const long long i = (long long)blockIdx.x * kScanSpan;
  const unsigned add = block_sums[blockIdx.x];
  for (int k = threadIdx.x; k < kScanSpan; k += blockDim.x)
    if (i + k < n) out[i + k] += add;
}

}  // namespace

size_t reg_scan_blocks(long long cells) { return static_cast<size_t>((cells + kScanSpan - 1) / kScanSpan); }

void launch_regularize(const Ctx& c, const RegDev& r, const RegBufs& b, cudaStream_t st) {
  if (c.n <= 0) return;
  const long long n = c.n;
  const unsigned blocks = static_cast<unsigned>((n + 255) / 256 < 65536 ? (n + 255) / 256 : 65536);
  cudaMemsetAsync(b.count, 0, sizeof(unsigned) * r.cells, st);
  cudaMemsetAsync(b.cursor, 0, sizeof(unsigned) * r.cells, st);
  cudaMemsetAsync(b.largest, 0, sizeof(unsigned) * c.nscenes, st);
  k_reg_count<<<blocks, 256, 0, st>>>(c, r, b.cell_of, b.target, b.inv_mass, b.count);
  const unsigned nb = static_cast<unsigned>(reg_scan_blocks(r.cells));
  k_scan_blocks<<<nb, kScanThreads, 0, st>>>(b.count, r.cells, b.start, b.block_sums);
  k_scan_top<<<1, kScanThreads, 0, st>>>(b.block_sums, static_cast<int>(nb));
  k_scan_add<<<nb, 256, 0, st>>>(b.start, r.cells, b.block_sums);
  k_reg_scatter<<<blocks, 256, 0, st>>>(c, b.cell_of, b.start, b.cursor, b.target, b.inv_mass, b.sorted,
                                        b.pos_sorted, b.inv_sorted, b.mat_sorted);
  k_reg_pairs<<<blocks, 256, 0, st>>>(c, r, b.cell_of, b.start, b.count, b.sorted, b.pos_sorted, b.inv_sorted,
                                      b.mat_sorted, b.shift, b.largest);
  k_reg_apply<<<blocks, 256, 0, st>>>(c, r, b.shift, b.largest);
}

}  // namespace mpm
