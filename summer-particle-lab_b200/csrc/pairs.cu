// Particle-pair passes over a cell sort of the particles: the solid position regularisation
// (src/three/solid-sampling.js:5-42, regularizeSolids; the reference's GPU twin is
// gpu/solver.py:565-648) and the particle-pair heat exchange with the enthalpy phase change
// (src/thermal.js:35-56, src/three/phase-change.js:12-18; GPU twin gpu/solver.py:775-811).
//
// Regularisation pass:
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
#include "pairs.h"

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

// ---- particle-pair heat exchange -------------------------------------------------------------
// k_heat_count / scan / k_heat_scatter: cell sort (cells one radius wide) with a packed copy of
//   position, temperature, conductivity and heat capacity in cell order
// k_heat_budget: per particle the sum of its conductances g over pairs (eps < r < radius), and its
//   budget min(1, 0.45 m cp / (dt sum g)) (1 without contacts)
// k_heat_flow: per particle heat_i = sum_j (T_j - T_i) g dt min(b_i, b_j) — each pair's +Q / -Q
//   gathered from both sides — then the enthalpy update, ambient loss and phase decode of the
//   particle; |Q| summed over pairs (each seen twice: halved) in FP64.

__global__ void k_heat_count(Ctx c, HeatDev hd, unsigned* cell_of, unsigned* count) {
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < c.n; h += (long long)gridDim.x * blockDim.x) {
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, h);
    const SceneDev& sc = c.scenes[s];
    const RegScene& rs = hd.scenes[s];
    float x[3];
    position(c.p, h, sc, x);
    int cc[3];
    for (int a = 0; a < 3; ++a) cc[a] = min(rs.nc[a] - 1, max(0, static_cast<int>(floorf(x[a] * hd.inv_hc))));
    const unsigned cell = static_cast<unsigned>(rs.cell_base + ((long long)cc[2] * rs.nc[1] + cc[1]) * rs.nc[0] + cc[0]);
    cell_of[h] = cell;
    atomicAdd(&count[cell], 1u);
  }
}

__global__ void k_heat_scatter(Ctx c, const unsigned* cell_of, const unsigned* start, unsigned* cursor, unsigned* sorted,
                               uint4* pos_sorted, float2* prop_sorted) {
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < c.n; h += (long long)gridDim.x * blockDim.x) {
    const unsigned cell = cell_of[h];
    const unsigned k = start[cell] + atomicAdd(&cursor[cell], 1u);
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, h);
    const int mi = c.single_material ? c.scenes[s].mat_base : c.p.mat[h];
    sorted[k] = static_cast<unsigned>(h);
    pos_sorted[k] = make_uint4(c.p.qx[h], c.p.qy[h], c.p.qz[h], __float_as_uint(c.p.T[h]));
    prop_sorted[k] = make_float2(c.mats_ext[mi].conductivity, c.p.m[h] * c.mats[mi].cp);
  }
}

// Visits the neighbours j of sorted particle ks within (eps, radius): fn(k, g) with the pair's
// conductance g = (1 - r / radius) geometry heat_rate 2 k_i k_j / (k_i + k_j).
template <typename Fn>
__device__ __forceinline__ void heat_pairs(const Ctx& c, const HeatDev& hd, const unsigned* cell_of,
                                           const unsigned* start, const unsigned* count, const uint4* pos_sorted,
                                           const float2* prop_sorted, long long ks, unsigned i, Fn&& fn) {
  const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, i);
  const SceneDev& sc = c.scenes[s];
  const RegScene& rs = hd.scenes[s];
  const uint4 pi = pos_sorted[ks];
  const float ki = prop_sorted[ks].x;
  const float to_m = sc.H * kInvFixedOne;
  const long long local = (long long)cell_of[i] - rs.cell_base;
  const int cx = static_cast<int>(local % rs.nc[0]), cy = static_cast<int>((local / rs.nc[0]) % rs.nc[1]),
            cz = static_cast<int>(local / ((long long)rs.nc[0] * rs.nc[1]));
  for (int z = max(0, cz - 1); z <= min(rs.nc[2] - 1, cz + 1); ++z)
    for (int y = max(0, cy - 1); y <= min(rs.nc[1] - 1, cy + 1); ++y)
      for (int x = max(0, cx - 1); x <= min(rs.nc[0] - 1, cx + 1); ++x) {
        const long long cell = rs.cell_base + ((long long)z * rs.nc[1] + y) * rs.nc[0] + x;
        const unsigned b = start[cell], e = b + count[cell];
        for (unsigned k = b; k < e; ++k) {
          if (k == ks) continue;
          const uint4 pj = pos_sorted[k];
          const float dx = static_cast<float>(static_cast<int>(pi.x - pj.x)) * to_m;
          const float dy = static_cast<float>(static_cast<int>(pi.y - pj.y)) * to_m;
          const float dz = static_cast<float>(static_cast<int>(pi.z - pj.z)) * to_m;
          const float r = sqrtf(dx * dx + dy * dy + dz * dz);
          if (!(r > hd.eps && r < hd.radius)) continue;
          const float kj = prop_sorted[k].x;
          const float kh = ki + kj > 0.f ? 2.f * ki * kj / (ki + kj) : 0.f;
          fn(k, (1.f - r / hd.radius) * hd.geom_rate * kh);
        }
      }
}

__global__ void k_heat_budget(Ctx c, HeatDev hd, const unsigned* cell_of, const unsigned* start, const unsigned* count,
                              const unsigned* sorted, const uint4* pos_sorted, const float2* prop_sorted, float* budget) {
  for (long long ks = blockIdx.x * (long long)blockDim.x + threadIdx.x; ks < c.n; ks += (long long)gridDim.x * blockDim.x) {
    const unsigned i = sorted[ks];
    double gsum = 0.0;
    heat_pairs(c, hd, cell_of, start, count, pos_sorted, prop_sorted, ks, i, [&](unsigned, float g) { gsum += g; });
    const double mcp = prop_sorted[ks].y;
    budget[ks] = gsum > 0.0 ? static_cast<float>(fmin(1.0, 0.45 * mcp / (hd.dt * gsum))) : 1.f;
  }
}

__global__ void k_heat_flow(Ctx c, HeatDev hd, const unsigned* cell_of, const unsigned* start, const unsigned* count,
                            const unsigned* sorted, const uint4* pos_sorted, const float2* prop_sorted,
                            const float* budget, double* exchanged) {
  double absq = 0.0;
  for (long long ks = blockIdx.x * (long long)blockDim.x + threadIdx.x; ks < c.n; ks += (long long)gridDim.x * blockDim.x) {
    const unsigned i = sorted[ks];
    const double Ti = __uint_as_float(pos_sorted[ks].w);
    const float bi = budget[ks];
    double heat = 0.0;
    heat_pairs(c, hd, cell_of, start, count, pos_sorted, prop_sorted, ks, i, [&](unsigned k, float g) {
      const double q = ((double)__uint_as_float(pos_sorted[k].w) - Ti) * g * hd.dt * fminf(bi, budget[k]);
      heat += q;
      absq += fabs(q);
    });
    // enthalpy update, ambient loss and the phase decode (src/thermal.js:51-55,
    // src/three/phase-change.js:12-18, src/three/simulation.js:260-270)
    const int s = c.nscenes == 1 ? 0 : find_scene_by_particle(c.scenes, c.nscenes, i);
    const int mi = c.single_material ? c.scenes[s].mat_base : c.p.mat[i];
    const MaterialExt& xt = c.mats_ext[mi];
    const double cp = c.mats[mi].cp, L = xt.latent;
    double hh = cp * Ti + (double)c.p.latent[i] * L + heat / c.p.m[i];
    if (hd.ambient) hh -= (Ti - hd.ambient_T) * cp * hd.dt * hd.ambient_rate;
    const unsigned char was = c.p.melted[i];
    unsigned char liquid = 0;
    double T;
    float f = 0.f;
    if (L > 0.0) {
      const double st = cp * xt.melting_point, en = st + L;
      if (hh <= st) { T = hh / cp; }
      else if (hh >= en) { T = (hh - L) / cp; f = 1.f; liquid = 1; }
      else { T = xt.melting_point; f = static_cast<float>((hh - st) / L); liquid = was; }
    } else {
      T = cp > 0.0 ? hh / cp : Ti;
    }
    c.p.T[i] = static_cast<float>(T);
    c.p.latent[i] = f;
    if (liquid != was) {
      // MPM3.resetParticle on a phase switch; a molten particle is released (Simulation3.pin(i, false))
      c.p.melted[i] = liquid;
      for (int e = 0; e < 9; ++e) {
        c.p.Cc[e][i] = 0.f;
        c.p.Dc[e][i] = 0.f;
      }
      c.p.ep[i] = 0.f;
      c.p.aux[i] = 0.f;
      if (liquid) c.p.pinned[i] = 0;
    }
  }
  // each pair was seen from both sides
  for (int o = 16; o > 0; o >>= 1) absq += __shfl_xor_sync(0xffffffffu, absq, o);
  if ((threadIdx.x & 31) == 0 && absq != 0.0) atomicAdd(exchanged, 0.5 * absq);
}

}  // namespace

void launch_exchange_heat(const Ctx& c, const HeatDev& hd, const HeatBufs& b, cudaStream_t st) {
  if (c.n <= 0) return;
  const long long n = c.n;
  const unsigned blocks = static_cast<unsigned>((n + 255) / 256 < 65536 ? (n + 255) / 256 : 65536);
  cudaMemsetAsync(b.count, 0, sizeof(unsigned) * hd.cells, st);
  cudaMemsetAsync(b.cursor, 0, sizeof(unsigned) * hd.cells, st);
  cudaMemsetAsync(b.exchanged, 0, sizeof(double), st);
  k_heat_count<<<blocks, 256, 0, st>>>(c, hd, b.cell_of, b.count);
  const unsigned nb = static_cast<unsigned>(reg_scan_blocks(hd.cells));
  k_scan_blocks<<<nb, kScanThreads, 0, st>>>(b.count, hd.cells, b.start, b.block_sums);
  k_scan_top<<<1, kScanThreads, 0, st>>>(b.block_sums, static_cast<int>(nb));
  k_scan_add<<<nb, 256, 0, st>>>(b.start, hd.cells, b.block_sums);
  k_heat_scatter<<<blocks, 256, 0, st>>>(c, b.cell_of, b.start, b.cursor, b.sorted, b.pos_sorted, b.prop_sorted);
  k_heat_budget<<<blocks, 256, 0, st>>>(c, hd, b.cell_of, b.start, b.count, b.sorted, b.pos_sorted, b.prop_sorted,
                                        b.budget);
  k_heat_flow<<<blocks, 256, 0, st>>>(c, hd, b.cell_of, b.start, b.count, b.sorted, b.pos_sorted, b.prop_sorted,
                                      b.budget, b.exchanged);
}

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
