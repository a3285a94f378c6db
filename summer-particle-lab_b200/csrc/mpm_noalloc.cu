// Allocation-free P2G entry point (mpm_p2g_noalloc in include/mpm_b200.h).
//
// Some callers cannot allocate device memory themselves: a host application that owns every device
// byte through its own pool and hands this library only the buffers it already holds (a Node addon
// fed by another GPU runtime, an engine with a fixed memory budget), or code running where a
// cudaMalloc is not allowed. For them this entry point performs the particle-to-grid transfer of
// the MLS-MPM step using caller-owned input and output buffers only. Its one intermediate, the grid
// accumulator, is a file-scope device array of fixed size instead of an allocation, so the call
// itself never allocates or frees device memory.
//
// The scratch array is kNoAllocMaxNodes nodes x 2 float4 = 8 MiB per GPU that loads the library and
// lives until the process exits. Every call shares it and it keeps the previous call's contents:
// each call clears the nodes it uses before scattering, and calls that overlap on the GPU (on
// different streams, or from several threads) race on it. Each call looks up the array's device
// address for the current device; the first call on a device may also load the library's device
// code there, so make it before any stream capture on that device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "mpm_b200.h"
#include "mpm_math.h"

namespace {

constexpr long long kNoAllocMaxNodes = 1ll << 18;  // 262,144 nodes, e.g. a 64^3-node grid

// (m, px, py, pz) and (fx, fy, fz, unused) per node
static __device__ __align__(256) float4 g_noalloc_grid[2 * kNoAllocMaxNodes];

struct NaGrid {
  double origin[3];
  float invH, H;
  int dims[3];
  float gravity[3];
};

__device__ __forceinline__ void stencil_fixed(double x, double origin, double invH, int dim, int& base, float& t) {
  // the same fixed-point position as the handle path's upload (22 fractional bits in cell units)
  const double qd = rint((x - origin) * invH * 4194304.0);
  const double hi = (double)(((long long)dim - 1) << 22);
  const unsigned q = (unsigned)fmin(fmax(qd, 0.0), hi);
  int b = (q < (1u << 21)) ? -1 : (int)((q - (1u << 21)) >> 22);
  b = min(max(b, 0), dim - 3);
  base = b;
  t = (float)((long long)q - ((long long)b << 22)) * 2.384185791015625e-07f;
}

__global__ void k_noalloc_clear(float4* grid, long long nodes) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 2 * nodes; i += (long long)gridDim.x * blockDim.x)
    grid[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Atomic P2G of one particle per thread (src/three/mpm.js:66-85, stress from F without a return as
// updateStress does for an uncached particle, src/three/mpm.js:33-37), dt-free channels.
__global__ void k_noalloc_p2g(float4* grid, NaGrid g, mpm::MaterialDev mt, long long n, const double* x, const float* v,
                              const double* F, const float* C, const float* m, const float* V) {
  const long long nodes = (long long)g.dims[0] * g.dims[1] * g.dims[2];
  const double invH = 1.0 / (double)g.H;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    int b[3];
    float t[3], w[3][3];
    for (int a = 0; a < 3; ++a) {
      stencil_fixed(x[p * 3 + a], g.origin[a], invH, g.dims[a], b[a], t[a]);
      mpm::bspline_weights(t[a], w[a]);
    }
    float D[9];
    for (int e = 0; e < 9; ++e) D[e] = (float)(F[p * 9 + e] - ((e % 4 == 0) ? 1.0 : 0.0));
    const float mp = m[p], Vp = V[p];
    const mpm::ConstitutiveOut co = mpm::constitutive_update(mt, D, 0.f, 0.f, Vp / mp, false);
    const float mv[3] = {mp * v[p * 3], mp * v[p * 3 + 1], mp * v[p * 3 + 2]};
    float mC[9];
    for (int e = 0; e < 9; ++e) mC[e] = mp * g.H * C[p * 9 + e];
    const float s = -4.f * Vp * g.invH;
    const float s6[6] = {s * co.tau.xx, s * co.tau.yy, s * co.tau.zz, s * co.tau.xy, s * co.tau.xz, s * co.tau.yz};
    for (int kz = 0; kz < 3; ++kz)
      for (int ky = 0; ky < 3; ++ky)
        for (int kx = 0; kx < 3; ++kx) {
          const float dx = kx - t[0], dy = ky - t[1], dz = kz - t[2];
          const float wt = w[0][kx] * w[1][ky] * w[2][kz];
          const long long node = ((long long)(b[2] + kz) * g.dims[1] + (b[1] + ky)) * g.dims[0] + (b[0] + kx);
          float* a0 = reinterpret_cast<float*>(&grid[node]);
          float* a1 = reinterpret_cast<float*>(&grid[nodes + node]);
          atomicAdd(a0 + 0, wt * mp);
          atomicAdd(a0 + 1, wt * (mv[0] + mC[0] * dx + mC[1] * dy + mC[2] * dz));
          atomicAdd(a0 + 2, wt * (mv[1] + mC[3] * dx + mC[4] * dy + mC[5] * dz));
          atomicAdd(a0 + 3, wt * (mv[2] + mC[6] * dx + mC[7] * dy + mC[8] * dz));
          atomicAdd(a1 + 0, wt * (s6[0] * dx + s6[3] * dy + s6[4] * dz));
          atomicAdd(a1 + 1, wt * (s6[3] * dx + s6[1] * dy + s6[5] * dz));
          atomicAdd(a1 + 2, wt * (s6[4] * dx + s6[5] * dy + s6[2] * dz));
        }
  }
}

// Node mass and momentum including dt (stress force + m g), the quantities mpm_grid_debug returns.
__global__ void k_noalloc_out(const float4* grid, long long nodes, float dt, NaGrid g, double* mass, double* mom) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nodes; i += (long long)gridDim.x * blockDim.x) {
    const float4 a0 = grid[i], a1 = grid[nodes + i];
    mass[i] = a0.x;
    mom[i * 3 + 0] = (double)a0.y + (double)dt * ((double)a1.x + (double)a0.x * g.gravity[0]);
    mom[i * 3 + 1] = (double)a0.z + (double)dt * ((double)a1.y + (double)a0.x * g.gravity[1]);
    mom[i * 3 + 2] = (double)a0.w + (double)dt * ((double)a1.z + (double)a0.x * g.gravity[2]);
  }
}

}  // namespace

extern "C" int mpm_p2g_noalloc(const mpm_domain* domain, const mpm_material* material, int64_t n, const double* x,
                               const float* v, const double* F, const float* C, const float* m, const float* V,
                               double dt, double* mass, double* momentum, void* stream) {
  if (!domain || !material || n < 0) return MPM_ERR_INVALID_ARG;
  if (n > 0 && (!x || !v || !F || !C || !m || !V)) return MPM_ERR_INVALID_ARG;
  if (!mass || !momentum) return MPM_ERR_INVALID_ARG;
  const int model = material->model;
  if (model < 0 || model > 11) return MPM_ERR_UNSUPPORTED;
  if (!(material->mu > 0) || !(3 * material->lambda + 2 * material->mu > 0)) return MPM_ERR_INVALID_ARG;
  // grid geometry as mpm_create derives it (src/three/discretization.js:12-14)
  const double H = domain->cell_size;
  if (!(H > 0) || !std::isfinite(H)) return MPM_ERR_INVALID_ARG;
  NaGrid g;
  std::memset(&g, 0, sizeof g);
  for (int a = 0; a < 3; ++a) {
    if (!(domain->upper[a] - domain->lower[a] >= H)) return MPM_ERR_INVALID_ARG;
    g.origin[a] = std::floor(domain->lower[a] / H + 1e-9) * H - 2 * H;
    g.dims[a] = static_cast<int>(std::ceil((domain->upper[a] - g.origin[a]) / H - 1e-9)) + 3;
    g.gravity[a] = static_cast<float>(domain->gravity[a]);
  }
  if (domain->cubic) {
    const int mx = std::max(g.dims[0], std::max(g.dims[1], g.dims[2]));
    g.dims[0] = g.dims[1] = g.dims[2] = mx;
  }
  g.H = static_cast<float>(H);
  g.invH = static_cast<float>(1.0 / H);
  const long long nodes = (long long)g.dims[0] * g.dims[1] * g.dims[2];
  if (nodes > kNoAllocMaxNodes) return MPM_ERR_CAPACITY;  // grid larger than the fixed scratch
  // set-up with the caller's device current: the device address of the scratch array on that
  // device (in host code the array's name is only a host-side stand-in, not a device address). It
  // is looked up on every call rather than cached, so a context re-created after a device reset
  // (or a change of current device) never gets a stale address; the lookup allocates nothing.
  void* scratch = nullptr;
  if (cudaGetSymbolAddress(&scratch, g_noalloc_grid) != cudaSuccess || !scratch) return MPM_ERR_CUDA;
  float4* grid = static_cast<float4*>(scratch);
  mpm::MaterialDev mt{};
  mt.model = model;
  mt.mu = static_cast<float>(material->mu);
  mt.lam = static_cast<float>(material->lambda);
  mt.yield_stress = static_cast<float>(material->yield_stress);
  mt.hardening = static_cast<float>(material->hardening);
  mt.T_ref = static_cast<float>(material->T_ref);
  mt.inv_T_span = material->T_hot > material->T_ref ? static_cast<float>(1.0 / (material->T_hot - material->T_ref)) : 0.f;
  mt.hot_ratio = static_cast<float>(material->hot_ratio);
  mt.wave_modulus = static_cast<float>(material->lambda + 2 * material->mu);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_noalloc_clear<<<592, 256, 0, st>>>(grid, nodes);
  if (n > 0) {
    const long long blocks = (n + 255) / 256 < 65536 ? (n + 255) / 256 : 65536;
    k_noalloc_p2g<<<static_cast<unsigned>(blocks), 256, 0, st>>>(grid, g, mt, n, x, v, F, C, m, V);
  }
  k_noalloc_out<<<592, 256, 0, st>>>(grid, nodes, static_cast<float>(dt), g, mass, momentum);
  return cudaGetLastError() == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}
