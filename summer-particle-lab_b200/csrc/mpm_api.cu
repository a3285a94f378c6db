// C ABI of the B200-native MLS-MPM solid step: handle lifetime, buffers, stepping, diagnostics.
// Declarations and the reference interface each function replaces: include/mpm_b200.h.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mpm_b200.h"
#include "mpm_internal.h"
#include "surrogate_net.h"
#include "pairs.h"

using mpm::Ctx;
using mpm::MaterialDev;
using mpm::SceneDev;

namespace {

constexpr int kMaxMats = 256;
constexpr uint32_t kCheckpointMagic = 0x3242504du;  // "MPB2"
constexpr uint32_t kCheckpointVersion = 3;  // 2: home-slot id array saved; 3: aux (Jp / dilation) saved

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Carver {
  char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    off = align_up(off, 256);
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
};

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

}  // namespace

struct mpm_handle {
  std::string err;
  cudaStream_t stream = nullptr;
  // The tile sort after a scatter pass runs on `side` beside the next substep's k_begin and grid
  // update; `main_ev` orders it after the pass, `side_ev` orders the next pass after it.
  cudaStream_t side = nullptr;
  cudaEvent_t main_ev = nullptr, side_ev = nullptr;
  bool side_pending = false;
  int num_sms = 148;
  mpm_domain dom{};
  SceneDev scene{};                  // scene 0 (the only scene of a single-scene handle)
  std::vector<SceneDev> scenes;      // every scene, in particle and grid order
  std::vector<int32_t> scene_material;  // batch handles: the material of each scene
  bool batch = false;                // created by mpm_batch_create
  cudaGraphExec_t graph = nullptr;   // captured substeps of mpm_batch_run
  int graph_substeps = 0;
  const unsigned* graph_parity = nullptr;  // particle buffer current when the graph was captured
  int64_t launches_per_graph = 0;
  std::vector<mpm_material> mats_host;
  std::vector<MaterialDev> mats_dev;
  std::vector<mpm::MaterialExt> mats_ext;
  std::vector<char> mat_set;
  int64_t cap = 0;
  int64_t n = 0;
  bool uploaded = false;
  bool grid_valid = false;   // acc[step_index & 1] holds the scatter of the current state
  bool pending_grid = false; // a scatter sits in acc[step_index & 1] (valid or stale)
  int use_tma = 1;
  int last_estimate = 0;           // substeps the last requested-dt call took (0: query the CFL dt first)
  double last_dt_requested = 0;
  // device memory
  void* pblock = nullptr;  size_t pblock_bytes = 0;   // particle arrays (current home order)
  void* pblock_alt = nullptr;                           // the other buffer of the permutation pass
  void* sblock = nullptr;                               // key and perm (shared by both buffers)
  mpm::Particles palt{};
  bool reorder_pending = false;   // permute into tile order at the next grid preparation
  int reorder_interval = 32;      // substeps between permutation passes (0: only at upload)
  int64_t substeps_since_reorder = 0;
  void* gblock = nullptr;  size_t gblock_bytes = 0;   // grid + sort + control
  void* snap = nullptr;    bool snap_valid = false;  int64_t snap_n = 0;
  void* staging = nullptr; size_t staging_bytes = 0;
  void** dptr_table = nullptr;                          // 12 device pointers for conversion
  double* ledger_partials = nullptr;
  double* ledger_out = nullptr;
  mpm::Ctrl* host_ctrl = nullptr;                        // pinned readback
  double* host_ledger = nullptr;                         // pinned readback
  Ctx ctx{};
  int g2p2g_blocks = 0, p2g_blocks = 0, grid_blocks = 0;
  int ws_blocks = 0;  // warp-specialised scatter passes available (CTAs), 0: not available
  // solid position regularisation: parameters and scratch (cells, sort, shifts), built on use
  mpm_regularizer reg{};
  void* rblock = nullptr;  size_t rblock_bytes = 0;
  mpm::RegBufs rbufs{};
  mpm::RegDev rdev{};
  bool reg_dirty = true;   // domain, scenes or spacing changed since the scratch was laid out
  // particle-pair heat exchange scratch, laid out for heat_radius
  void* hblock = nullptr;  size_t hblock_bytes = 0;
  mpm::HeatBufs hbufs{};
  mpm::HeatDev hdev{};
  double heat_radius = 0;
  double* host_exchanged = nullptr;  // pinned readback
  int slab_planes = 0;     // batch of slabs along z: node planes shared by consecutive scenes
  // learned return mode: the network's BF16 tensor-core weights, its FP32 parameters and the gate
  // counts, one device block owned by the handle (a copy: the surrogate may be destroyed after)
  int return_mode = MPM_RETURN_EXACT;
  void* mlp_block = nullptr;
  // profiling: event pairs around launches while enabled
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, int>> ev_used;  // (kernel id, index of the start event in ev_pool)
  size_t ev_next = 0;
  int64_t launches = 0;
};

// Records a CUDA event pair around one launch when profiling is on.
struct ProfScope {
  mpm_handle* h;
  int id;
  size_t idx = 0;
  bool on;
  cudaStream_t st;
  ProfScope(mpm_handle* hh, int kid, cudaStream_t s = nullptr) : h(hh), id(kid), on(hh->profiling), st(s ? s : hh->stream) {
    ++h->launches;
    if (!on) return;
    if (h->ev_next + 2 > h->ev_pool.size()) {
      for (int k = 0; k < 256; ++k) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        h->ev_pool.push_back(e);
      }
    }
    idx = h->ev_next;
    h->ev_next += 2;
    cudaEventRecord(h->ev_pool[idx], st);
  }
  ~ProfScope() {
    if (!on) return;
    cudaEventRecord(h->ev_pool[idx + 1], st);
    h->ev_used.push_back({id, static_cast<int>(idx)});
  }
};

#define MPM_CUDA(h, call)                                                          \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      (h)->err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
      return e_ == cudaErrorMemoryAllocation ? MPM_ERR_OUT_OF_MEMORY : MPM_ERR_CUDA; \
    }                                                                              \
  } while (0)

static void drop_graph(mpm_handle* h) {
  if (h->graph) cudaGraphExecDestroy(h->graph);
  h->graph = nullptr;
  h->graph_substeps = 0;
}

static int fail(mpm_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

// Scene geometry from the domain (src/three/discretization.js:12-14) and the node thresholds the
// grid update uses, computed in double exactly as the reference compares q < lower + h.
static int build_scene(mpm_handle* h, const mpm_domain& d, SceneDev& s) {
  const double H = d.cell_size;
  if (!(H > 0) || !std::isfinite(H)) return fail(h, MPM_ERR_INVALID_ARG, "cell_size must be positive");
  int dims[3];
  double origin[3];
  for (int a = 0; a < 3; ++a) {
    if (!std::isfinite(d.lower[a]) || !std::isfinite(d.upper[a]) || !(d.upper[a] - d.lower[a] >= H))
      return fail(h, MPM_ERR_INVALID_ARG, "domain must span at least one cell on every axis");
    origin[a] = std::floor(d.lower[a] / H + 1e-9) * H - 2 * H;
    dims[a] = static_cast<int>(std::ceil((d.upper[a] - origin[a]) / H - 1e-9)) + 3;
  }
  if (d.cubic) {
    const int m = std::max(dims[0], std::max(dims[1], dims[2]));
    dims[0] = dims[1] = dims[2] = m;
  }
  std::memset(&s, 0, sizeof s);
  s.H = static_cast<float>(H);
  s.invH = static_cast<float>(1.0 / H);
  for (int a = 0; a < 3; ++a) {
    if (dims[a] > 1023 || dims[a] < 4) return fail(h, MPM_ERR_INVALID_ARG, "grid must have 4..1023 nodes per axis");
    s.dims[a] = dims[a];
    s.tiles[a] = ((dims[a] - 3) >> 2) + 1;
    s.gdim[a] = 4 * s.tiles[a] + 4;
    s.ntiles[a] = s.gdim[a] / 4;
    s.origin[a] = origin[a];
    int lo = -1, hi = dims[a];
    for (int i = 0; i < dims[a]; ++i) {
      const double q = origin[a] + i * H;
      if (q < d.lower[a] + H) lo = i;
      if (q > d.upper[a] - H && hi == dims[a]) hi = i;
    }
    s.wall_lo[a] = lo;
    s.wall_hi[a] = hi;
    const double clo = d.lower[a] + 1e-6 * H, chi = d.upper[a] - 1e-6 * H;
    const double qmax = static_cast<double>((static_cast<long long>(dims[a]) - 1) << mpm::kFracBits);
    s.qlo[a] = static_cast<unsigned>(std::min(qmax, std::max(0.0, std::ceil((clo - origin[a]) / H * 4194304.0))));
    s.qhi[a] = static_cast<unsigned>(std::min(qmax, std::max(0.0, std::floor((chi - origin[a]) / H * 4194304.0))));
    s.gravity[a] = static_cast<float>(d.gravity[a]);
  }
  s.clamp = d.clamp_positions ? 1 : 0;
  s.sticky = d.sticky_floor ? 1 : 0;
  s.mass_eps = static_cast<float>(d.mass_eps > 0 ? d.mass_eps : 1e-12);
  s.cfl = static_cast<float>(d.cfl > 0 ? d.cfl : 0.4);
  s.dt_max = static_cast<float>(d.dt_max > 0 ? d.dt_max : 3.0e38);
  s.grad_limit = static_cast<float>(d.grad_limit > 0 ? d.grad_limit : 0.08);
  s.node_base = 0;
  s.tile_base = 0;
  s.node_tile_base = 0;
  s.mat_base = 0;
  return MPM_OK;
}

static int free_device(mpm_handle* h) {
  if (h->pblock) cudaFree(h->pblock);
  if (h->pblock_alt) cudaFree(h->pblock_alt);
  if (h->sblock) cudaFree(h->sblock);
  h->pblock_alt = h->sblock = nullptr;
  if (h->gblock) cudaFree(h->gblock);
  if (h->snap) cudaFree(h->snap);
  if (h->staging) cudaFree(h->staging);
  if (h->dptr_table) cudaFree(h->dptr_table);
  if (h->ledger_partials) cudaFree(h->ledger_partials);
  if (h->rblock) cudaFree(h->rblock);
  h->rblock = nullptr;
  h->rblock_bytes = 0;
  h->reg_dirty = true;
  if (h->hblock) cudaFree(h->hblock);
  h->hblock = nullptr;
  h->hblock_bytes = 0;
  h->heat_radius = 0;
  if (h->host_exchanged) cudaFreeHost(h->host_exchanged);
  h->host_exchanged = nullptr;
  if (h->host_ctrl) cudaFreeHost(h->host_ctrl);
  if (h->host_ledger) cudaFreeHost(h->host_ledger);
  if (h->mlp_block) cudaFree(h->mlp_block);
  h->mlp_block = nullptr;
  h->return_mode = MPM_RETURN_EXACT;
  h->ctx.learned = 0;
  h->pblock = h->gblock = h->snap = h->staging = nullptr;
  h->dptr_table = nullptr;
  h->ledger_partials = nullptr;
  h->host_ctrl = nullptr;
  h->host_ledger = nullptr;
  return MPM_OK;
}

// Carve the particle arrays of capacity cap out of one allocation (or measure it with base null).
static size_t carve_particles(char* base, int64_t cap, mpm::Particles& p) {
  Carver c{base};
  p.qx = c.take<unsigned>(cap); p.qy = c.take<unsigned>(cap); p.qz = c.take<unsigned>(cap);
  p.vx = c.take<float>(cap); p.vy = c.take<float>(cap); p.vz = c.take<float>(cap);
  p.C = c.take<float>(cap * 9);
  p.D = c.take<float>(cap * 9);
  for (int e = 0; e < 9; ++e) {
    p.Cc[e] = p.C ? p.C + e * cap : nullptr;
    p.Dc[e] = p.D ? p.D + e * cap : nullptr;
  }
  p.m = c.take<float>(cap); p.V = c.take<float>(cap);
  p.ep = c.take<float>(cap); p.T = c.take<float>(cap);
  p.aux = c.take<float>(cap);
  p.latent = c.take<float>(cap);
  p.melted = c.take<unsigned char>(cap);
  p.mat = c.take<unsigned short>(cap);
  p.pinned = c.take<unsigned char>(cap);
  p.id = c.take<unsigned>(cap);
  p.cap = cap;
  return align_up(c.off, 256);
}

// Permutation pass: rewrite the state in sort order into the other buffer and make it current.
// The main stream waits for a tile sort still running on the side stream.
static void join_side(mpm_handle* h) {
  if (!h->side_pending) return;
  cudaStreamWaitEvent(h->stream, h->side_ev, 0);
  h->side_pending = false;
}

static int permute_state(mpm_handle* h) {
  join_side(h);
  h->ctx.n = h->n;
  mpm::launch_permute(h->ctx, h->palt, h->stream);
  MPM_CUDA(h, cudaGetLastError());
  std::swap(h->pblock, h->pblock_alt);
  mpm::Particles cur = h->palt;
  h->palt = h->ctx.p;
  h->ctx.p = cur;
  h->substeps_since_reorder = 0;
  return MPM_OK;
}

// Grid, sort buffers and control block of every scene in one allocation. Scene s owns nodes
// [node_base, node_base + gdim^3), particle tiles [tile_base, ...) and node tiles
// [node_tile_base, ...); bases increase with s, so a tile-sorted particle order keeps each
// scene's particles contiguous and in scene order.
static int alloc_grid(mpm_handle* h) {
  if (h->gblock) {
    cudaFree(h->gblock);
    h->gblock = nullptr;
  }
  const int ns = static_cast<int>(h->scenes.size());
  long long nodes = 0;
  int tiles = 0, ntiles = 0;
  for (SceneDev& s : h->scenes) {
    s.node_base = nodes;
    s.tile_base = tiles;
    s.node_tile_base = ntiles;
    nodes += (long long)s.gdim[0] * s.gdim[1] * s.gdim[2];
    tiles += s.tiles[0] * s.tiles[1] * s.tiles[2];
    ntiles += s.ntiles[0] * s.ntiles[1] * s.ntiles[2];
  }
  h->scene = h->scenes[0];
  const int scan_blocks = (tiles + 1 + 4095) / 4096;
  auto lay = [&](char* base, Ctx& c, void** tmaps, SceneDev** scenes, MaterialDev** mats) {
    Carver cv{base};
    for (int k = 0; k < 2; ++k) {
      c.g.acc0[k] = cv.take<float4>(nodes);
      c.g.acc1[k] = cv.take<float4>(nodes);
      c.g.heat[k] = cv.take<float>(nodes);
    }
    c.g.tnode = cv.take<float>(nodes);
    c.g.mnode = cv.take<float>(nodes);
    c.g.tile_epoch = cv.take<unsigned>(ntiles);
    c.g.vel = cv.take<float4>(nodes);
    c.g.tile_flag = cv.take<unsigned>(ntiles);
    c.g.active[0] = cv.take<unsigned>(ntiles);
    c.g.active[1] = cv.take<unsigned>(ntiles);
    c.s.count = cv.take<unsigned>(tiles + 1);
    c.s.start = cv.take<unsigned>(tiles + 1);
    c.s.block_off = cv.take<unsigned>(scan_blocks + 1);
    c.s.rank = cv.take<unsigned>(tiles + 1);
    c.s.block_rank = cv.take<unsigned>(scan_blocks + 1);
    c.s.work[0] = cv.take<uint4>(tiles);
    c.s.work[1] = cv.take<uint4>(tiles);
    c.ctrl = cv.take<mpm::Ctrl>(1);
    c.dt_scene = cv.take<float>(ns);
    c.wave_max = cv.take<unsigned>(ns);
    c.grad_max = cv.take<unsigned>(ns);
    c.time_scene = cv.take<double>(ns);
    *scenes = cv.take<SceneDev>(ns);
    *mats = cv.take<MaterialDev>(kMaxMats);
    c.mats_ext = cv.take<mpm::MaterialExt>(kMaxMats);
    *tmaps = cv.take<char>(128 * (size_t)ns);
    return align_up(cv.off, 256);
  };
  h->reg_dirty = true;  // neighbour cells follow the scenes' grids
  h->heat_radius = 0;
  Ctx probe{};
  void* t;
  SceneDev* sp;
  MaterialDev* mp;
  const size_t bytes = lay(nullptr, probe, &t, &sp, &mp);
  MPM_CUDA(h, cudaMalloc(&h->gblock, bytes));
  h->gblock_bytes = bytes;
  MPM_CUDA(h, cudaMemsetAsync(h->gblock, 0, bytes, h->stream));
  Ctx& c = h->ctx;
  void* tm;
  SceneDev* scenes;
  MaterialDev* mats;
  lay(static_cast<char*>(h->gblock), c, &tm, &scenes, &mats);
  c.scenes = scenes;
  c.mats = mats;
  c.nscenes = ns;
  c.total_tiles = tiles;
  c.total_node_tiles = ntiles;
  MPM_CUDA(h, cudaMemcpyAsync(scenes, h->scenes.data(), sizeof(SceneDev) * ns, cudaMemcpyHostToDevice, h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(mats, h->mats_dev.data(), sizeof(MaterialDev) * kMaxMats, cudaMemcpyHostToDevice,
                              h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<mpm::MaterialExt*>(c.mats_ext), h->mats_ext.data(),
                              sizeof(mpm::MaterialExt) * kMaxMats, cudaMemcpyHostToDevice, h->stream));
  // TMA descriptor of each scene's velocity grid: 4D {channel 4, x, y, z}, box {4, 6, 6, 6}, fp32.
  // A scene's grid starts at a float4 node (16-byte aligned) and its strides are multiples of 16 B.
  c.tmaps = nullptr;
  c.use_tma = 0;
  auto encode = tensor_map_encoder();
  if (encode && h->use_tma) {
    std::vector<CUtensorMap> maps(ns);
    bool ok = true;
    for (int k = 0; k < ns && ok; ++k) {
      const SceneDev& s = h->scenes[k];
      std::memset(&maps[k], 0, sizeof(CUtensorMap));
      cuuint64_t gdims[4] = {4, (cuuint64_t)s.gdim[0], (cuuint64_t)s.gdim[1], (cuuint64_t)s.gdim[2]};
      cuuint64_t gstrides[3] = {16, 16ull * s.gdim[0], 16ull * s.gdim[0] * s.gdim[1]};
      cuuint32_t box[4] = {4, mpm::kWinG, mpm::kWinG, mpm::kWinG};
      cuuint32_t estr[4] = {1, 1, 1, 1};
      CUresult r = encode(&maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, c.g.vel + s.node_base, gdims, gstrides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      ok = r == CUDA_SUCCESS;
    }
    if (ok) {
      static_assert(sizeof(CUtensorMap) == 128, "tensor map stride");
      MPM_CUDA(h, cudaMemcpyAsync(tm, maps.data(), sizeof(CUtensorMap) * ns, cudaMemcpyHostToDevice, h->stream));
      MPM_CUDA(h, cudaStreamSynchronize(h->stream));  // maps is a host temporary
      c.tmaps = tm;
      c.use_tma = 1;
    }
  }
  h->grid_valid = false;
  h->pending_grid = false;
  return MPM_OK;
}

// The gated instances of the particle pass (learned: the network's guess; newton: a guess from the
// initial flow stress) serve scenes without grid conduction and without the history laws (snow,
// sand, pressure); anything else runs the exact return map.
static void apply_return_mode(mpm_handle* h) {
  const bool eligible = h->mlp_block && !h->ctx.has_aux && !h->ctx.conduct;
  h->ctx.learned = eligible && h->return_mode == MPM_RETURN_LEARNED_GATED   ? 1
                   : eligible && h->return_mode == MPM_RETURN_NEWTON_GATED ? 2
                                                                             : 0;
}

static void refresh_flags(mpm_handle* h) {
  bool plastic = false, thermal = false, aux = false;
  for (size_t i = 0; i < h->mats_host.size(); ++i) {
    if (!h->mat_set[i]) continue;
    const int m = h->mats_host[i].model;
    if (m >= 2) plastic = true;
    if (m == 10) thermal = true;
    if (mpm::aux_model(m)) aux = true;
  }
  h->ctx.has_plastic = plastic ? 1 : 0;
  h->ctx.has_aux = aux ? 1 : 0;
  h->ctx.has_thermal = thermal || h->ctx.has_thermal ? 1 : 0;
  apply_return_mode(h);
}

// The error for the device status flags st (MPM_OK when none is set).
static int status_error(mpm_handle* h, unsigned st) {
  if (st & MPM_STATUS_TIMEOUT) return fail(h, MPM_ERR_TIMEOUT, "a bounded device wait gave up (TMA copy did not complete)");
  if (st & MPM_STATUS_NONFINITE) return fail(h, MPM_ERR_NONFINITE, "non-finite particle state");
  if (st & MPM_STATUS_INVALID_J) return fail(h, MPM_ERR_INVALID_J, "det F <= 0 in a particle");
  if (st & MPM_STATUS_OUT_OF_RANGE) return fail(h, MPM_ERR_OUT_OF_RANGE, "a particle left the grid");
  if (st & MPM_STATUS_SORT_MISMATCH) return fail(h, MPM_ERR_STATE, "tile sort keys and counts disagreed");
  return MPM_OK;
}

static int check_status(mpm_handle* h) {
  join_side(h);
  MPM_CUDA(h, cudaMemcpyAsync(h->host_ctrl, h->ctx.ctrl, sizeof(mpm::Ctrl), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  return status_error(h, h->host_ctrl->status);
}

// Counting sort of the current state by tile and the dt-free P2G into acc[step_index & 1].
static int prepare_grid(mpm_handle* h) {
  join_side(h);
  Ctx& c = h->ctx;
  c.n = h->n;
  if (h->pending_grid) {
    ProfScope ps(h, -1);
    mpm::launch_grid_clear(c, h->stream, h->grid_blocks);
    MPM_CUDA(h, cudaGetLastError());
  }
  { ProfScope ps(h, -1); mpm::launch_control_init(c, h->stream); }
  MPM_CUDA(h, cudaMemsetAsync(c.s.count, 0, sizeof(unsigned) * (c.total_tiles + 1), h->stream));
  { ProfScope ps(h, 6); mpm::launch_keys(c, h->stream); }
  { ProfScope ps(h, 3); mpm::launch_scan(c, h->stream, true); }
  { ProfScope ps(h, 4); mpm::launch_sort_scatter(c, h->stream, true); }
  if (h->reorder_pending) {
    ProfScope ps(h, -1);
    const int rc = permute_state(h);
    if (rc != MPM_OK) return rc;
    h->reorder_pending = false;
  }
  { ProfScope ps(h, 5); mpm::launch_p2g(h->ctx, h->stream, h->p2g_blocks); }
  if (h->slab_planes) { ProfScope ps(h, -1); mpm::launch_halo_sum(h->ctx, h->stream, h->slab_planes); }
  MPM_CUDA(h, cudaGetLastError());
  h->grid_valid = true;
  h->pending_grid = true;
  return MPM_OK;
}

// One substep: k_begin and the grid update (beside the previous pass's tile sort, if that is still
// running on the side stream), then the particle pass; a scatter pass forks its tile sort (scan +
// counting sort of the keys it wrote) onto the side stream, where it overlaps the next substep's
// k_begin and grid update. The two never touch the same data: the sort works on the keys, counts,
// perm and the work list of the pass's parity, k_begin and the grid update on the control block's
// step fields, the other list's counters and the grid.
static void launch_substep(mpm_handle* h, bool scatter) {
  Ctx& c = h->ctx;
  { ProfScope ps(h, 0); mpm::launch_begin(c, h->stream); }
  { ProfScope ps(h, 1); mpm::launch_grid_update(c, h->stream, h->grid_blocks); }
  if (c.conduct) {
    ProfScope ps(h, -1);
    mpm::launch_conduct(c, h->stream, h->grid_blocks);
  }
  join_side(h);
  { ProfScope ps(h, 2); mpm::launch_g2p2g(c, h->stream, h->g2p2g_blocks, scatter); }
  if (scatter && h->slab_planes) { ProfScope ps(h, -1); mpm::launch_halo_sum(c, h->stream, h->slab_planes); }
  if (scatter) {
    cudaEventRecord(h->main_ev, h->stream);
    cudaStreamWaitEvent(h->side, h->main_ev, 0);
    { ProfScope ps(h, 3, h->side); mpm::launch_scan(c, h->side, false); }
    { ProfScope ps(h, 4, h->side); mpm::launch_sort_scatter(c, h->side, false); }
    cudaEventRecord(h->side_ev, h->side);
    h->side_pending = true;
  }
}

MaterialDev mpm::material_to_device(const mpm_material& m) {
  MaterialDev d{};
  d.model = m.model;
  d.mu = static_cast<float>(m.mu);
  d.lam = static_cast<float>(m.lambda);
  d.yield_stress = static_cast<float>(m.yield_stress);
  d.hardening = static_cast<float>(m.hardening);
  d.T_ref = static_cast<float>(m.T_ref);
  d.inv_T_span = m.T_hot > m.T_ref ? static_cast<float>(1.0 / (m.T_hot - m.T_ref)) : 0.f;
  d.hot_ratio = static_cast<float>(m.hot_ratio);
  d.heat_per_work = m.specific_heat > 0 ? static_cast<float>(m.heat_fraction / m.specific_heat) : 0.f;
  d.cp = static_cast<float>(m.specific_heat);
  d.wave_modulus = static_cast<float>(m.lambda + 2 * m.mu);
  d.jc_n = static_cast<float>(m.jc_n);
  d.jc_C = static_cast<float>(m.jc_C);
  d.jc_inv_rate0 = m.jc_rate0 > 0 ? static_cast<float>(1.0 / m.jc_rate0) : 0.f;
  d.jc_inv_T_span = m.T_melt > m.T_ref ? static_cast<float>(1.0 / (m.T_melt - m.T_ref)) : 0.f;
  d.jc_m = static_cast<float>(m.jc_m);
  d.cr_on = m.creep_rate > 0 ? 1 : 0;
  d.cr_log_rate = m.creep_rate > 0 ? static_cast<float>(std::log(m.creep_rate)) : 0.f;
  d.cr_Q_over_R = static_cast<float>(m.creep_Q / 8.314462618);
  d.cr_T_offset = static_cast<float>(m.temperature_offset);
  d.cr_inv_Tref_abs = static_cast<float>(1.0 / (m.T_ref + m.temperature_offset));
  d.cr_n = static_cast<float>(m.creep_n);
  d.cr_inv_stress = m.creep_stress > 0 ? static_cast<float>(1.0 / m.creep_stress) : 0.f;
  return d;
}

static mpm::MaterialExt to_device_ext(const mpm_material& m) {
  mpm::MaterialExt d{};
  d.snow_lo = static_cast<float>(-m.yield_strain);
  d.snow_hi = static_cast<float>(0.3 * m.yield_strain);
  const double sn = std::sin(m.friction_deg * 3.14159265358979323846 / 180.0);
  d.sand_k = static_cast<float>(std::sqrt(2.0 / 3.0) * 2 * sn / (3 - sn) * (3 * m.lambda + 2 * m.mu) / (2 * m.mu));
  d.bulk = static_cast<float>(m.lambda + 2 * m.mu / 3);
  d.dp_c = static_cast<float>(m.dp_cohesion);
  d.dp_a = static_cast<float>(m.dp_slope);
  d.dp_b = static_cast<float>(m.dp_dilatancy);
  d.dp_T = static_cast<float>(m.dp_tension);
  d.df_a2 = static_cast<float>(m.df_alpha * m.df_alpha);
  d.df_B = static_cast<float>(1 + m.df_alpha * m.df_alpha / 9);
  d.df_plateau = static_cast<float>(m.df_plateau);
  d.df_gamma = static_cast<float>(m.df_gamma);
  d.df_densify = static_cast<float>(m.df_densify);
  d.df_beta = static_cast<float>(m.df_beta);
  d.df_inv_epsd = m.df_eps_d > 0 ? static_cast<float>(1.0 / m.df_eps_d) : 0.f;
  d.conductivity = static_cast<float>(m.conductivity);
  d.melting_point = static_cast<float>(m.melting_point);
  d.latent = m.latent_heat > 0 ? static_cast<float>(m.latent_heat) : 0.f;
  return d;
}

static int validate_material(const mpm_material* m, std::string& why) {
  if (!m) { why = "material is null"; return MPM_ERR_INVALID_ARG; }
  if (m->model < 0 || m->model > 11) {
    why = "material model not built (supported: 0-11)";
    return MPM_ERR_UNSUPPORTED;
  }
  if (!(m->mu > 0) || !(3 * m->lambda + 2 * m->mu > 0) || !std::isfinite(m->mu) || !std::isfinite(m->lambda)) {
    why = "moduli must satisfy mu > 0 and 3 lambda + 2 mu > 0";
    return MPM_ERR_INVALID_ARG;
  }
  if (m->model >= 4 && (!(m->yield_stress >= 0) || !(m->hardening >= 0))) {
    why = "yield stress and hardening must be non-negative";
    return MPM_ERR_INVALID_ARG;
  }
  if (m->model == 10 && !(m->T_hot > m->T_ref)) {
    why = "T_hot must exceed T_ref";
    return MPM_ERR_INVALID_ARG;
  }
  if ((m->model == 6 || m->model == 7) && (!(m->jc_rate0 > 0) || !(m->jc_n >= 0) || !(m->jc_C >= 0))) {
    why = "Johnson-Cook needs rate0 > 0, n >= 0 and C >= 0";
    return MPM_ERR_INVALID_ARG;
  }
  if (m->model == 6 && (!(m->T_melt > m->T_ref) || !(m->jc_m >= 0))) {
    why = "Johnson-Cook model 6 needs T_melt > T_ref and m >= 0";
    return MPM_ERR_INVALID_ARG;
  }
  if (m->model == 11 && (!(m->creep_rate >= 0) || !(m->creep_stress > 0) || !(m->T_ref + m->temperature_offset > 0))) {
    why = "Norton creep needs rate >= 0, stress > 0 and an absolute reference temperature > 0";
    return MPM_ERR_INVALID_ARG;
  }
  if (m->model == 2 && !(m->yield_strain > 0 && m->yield_strain < 1)) {
    why = "snow needs 0 < yield_strain < 1";
    return MPM_ERR_INVALID_ARG;
  }
  if (m->model == 3 && !(m->friction_deg > 0 && m->friction_deg < 90)) {
    why = "sand needs a friction angle in (0, 90) degrees";
    return MPM_ERR_INVALID_ARG;
  }
  // src/three/pressure-plasticity.js:2-10: the reference's limits on the dimensionless
  // parameters, non-negative strengths, dilatancy <= slope and slope * tension <= cohesion
  if (m->model == 8 && (!(m->dp_cohesion >= 0) || !(m->dp_slope >= 0 && m->dp_slope <= 2) ||
                        !(m->dp_dilatancy >= 0 && m->dp_dilatancy <= m->dp_slope) || !(m->dp_tension >= 0) ||
                        !(m->dp_slope * m->dp_tension <= m->dp_cohesion * (1 + 1e-12) + 1e-300))) {
    why = "cohesive Drucker-Prager needs cohesion, tension >= 0, 0 <= dilatancy <= slope <= 2 and slope * tension <= cohesion";
    return MPM_ERR_INVALID_ARG;
  }
  if (m->model == 9 && (!(m->df_alpha >= 0.05 && m->df_alpha <= std::sqrt(4.5)) || !(m->df_plateau > 0) ||
                        !(m->df_gamma >= 0) || !(m->df_densify > 0) || !(m->df_beta >= 1 && m->df_beta <= 5) ||
                        !(m->df_eps_d >= 0.05 && m->df_eps_d <= 3))) {
    why = "Deshpande-Fleck foam needs alpha in [0.05, sqrt(4.5)], plateau, densify > 0, gamma >= 0, beta in [1, 5], eps_D in [0.05, 3]";
    return MPM_ERR_INVALID_ARG;
  }
  // src/three/phase-change.js:4-9 (melting point in [-100, 2000], latent heat in [1000, 2e6] when
  // enabled) in the caller's units; here: finite, latent heat >= 0, conductivity >= 0
  if (!(m->conductivity >= 0) || !std::isfinite(m->conductivity) || !(m->latent_heat >= 0) ||
      !std::isfinite(m->latent_heat) || !std::isfinite(m->melting_point)) {
    why = "conductivity and latent heat must be finite and >= 0, the melting point finite";
    return MPM_ERR_INVALID_ARG;
  }
  if (m->latent_heat > 0 && !(m->specific_heat > 0)) {
    why = "phase change needs a specific heat > 0";
    return MPM_ERR_INVALID_ARG;
  }
  if (m->heat_fraction < 0 || m->heat_fraction > 1) {
    why = "heat_fraction must lie in [0, 1]";
    return MPM_ERR_INVALID_ARG;
  }
  return MPM_OK;
}

extern "C" {

int mpm_abi_version(void) { return MPM_ABI_VERSION; }

int mpm_validate_material(const mpm_material* material) {
  std::string why;
  return validate_material(material, why);
}

const char* mpm_error_string(int status) {
  switch (status) {
    case MPM_OK: return "ok";
    case MPM_ERR_INVALID_ARG: return "invalid argument";
    case MPM_ERR_OUT_OF_MEMORY: return "out of device memory";
    case MPM_ERR_CUDA: return "CUDA error";
    case MPM_ERR_NONFINITE: return "non-finite particle state";
    case MPM_ERR_INVALID_J: return "det F <= 0";
    case MPM_ERR_OUT_OF_RANGE: return "particle outside the grid";
    case MPM_ERR_TIMEOUT: return "bounded device wait timed out";
    case MPM_ERR_STATE: return "call out of order";
    case MPM_ERR_CAPACITY: return "capacity exceeded";
    case MPM_ERR_UNSUPPORTED: return "unsupported material model";
    default: return "unknown status";
  }
}

int mpm_create(const mpm_domain* domain, int64_t capacity, mpm_handle** out) {
  if (!out || !domain || capacity <= 0 || capacity > (int64_t)1 << 31) return MPM_ERR_INVALID_ARG;
  *out = nullptr;
  mpm_handle* h = new mpm_handle();
  SceneDev s;
  int rc = build_scene(h, *domain, s);
  if (rc != MPM_OK) {
    delete h;
    return rc;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    delete h;
    return MPM_ERR_CUDA;
  }
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return MPM_ERR_CUDA;
  }
  if (cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->main_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->side_ev, cudaEventDisableTiming) != cudaSuccess) {
    if (h->main_ev) cudaEventDestroy(h->main_ev);
    if (h->side) cudaStreamDestroy(h->side);
    cudaStreamDestroy(h->stream);
    delete h;
    return MPM_ERR_CUDA;
  }
  h->dom = *domain;
  h->scene = s;
  h->scenes.assign(1, s);
  h->cap = capacity;
  h->use_tma = std::getenv("MPM_B200_NO_TMA") ? 0 : 1;  // plain-load gather window when set
  h->mats_host.assign(kMaxMats, mpm_material{});
  h->mats_dev.assign(kMaxMats, MaterialDev{});
  h->mats_ext.assign(kMaxMats, mpm::MaterialExt{});
  h->mat_set.assign(kMaxMats, 0);
  mpm::Particles p{};
  const size_t pbytes = carve_particles(nullptr, capacity, p);
  auto bail = [&](int code) {
    free_device(h);
    cudaEventDestroy(h->main_ev);
    cudaEventDestroy(h->side_ev);
    cudaStreamDestroy(h->side);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return code;
  };
  if (cudaMalloc(&h->pblock, pbytes) != cudaSuccess) return bail(MPM_ERR_OUT_OF_MEMORY);
  if (cudaMalloc(&h->pblock_alt, pbytes) != cudaSuccess) return bail(MPM_ERR_OUT_OF_MEMORY);
  if (cudaMalloc(&h->sblock, 2 * capacity * sizeof(unsigned) + 512) != cudaSuccess) return bail(MPM_ERR_OUT_OF_MEMORY);
  h->pblock_bytes = pbytes;
  carve_particles(static_cast<char*>(h->pblock), capacity, h->ctx.p);
  carve_particles(static_cast<char*>(h->pblock_alt), capacity, h->palt);
  h->ctx.p.key = h->palt.key = static_cast<unsigned*>(h->sblock);
  h->ctx.p.perm = h->palt.perm = static_cast<unsigned*>(h->sblock) + align_up(capacity, 64);
  if (cudaMemsetAsync(h->pblock, 0, pbytes, h->stream) != cudaSuccess) return bail(MPM_ERR_CUDA);
  if (cudaMemsetAsync(h->pblock_alt, 0, pbytes, h->stream) != cudaSuccess) return bail(MPM_ERR_CUDA);
  if (cudaMalloc(reinterpret_cast<void**>(&h->dptr_table), 16 * sizeof(void*)) != cudaSuccess) return bail(MPM_ERR_OUT_OF_MEMORY);
  if (cudaMallocHost(reinterpret_cast<void**>(&h->host_ctrl), sizeof(mpm::Ctrl)) != cudaSuccess) return bail(MPM_ERR_OUT_OF_MEMORY);
  if (cudaMallocHost(reinterpret_cast<void**>(&h->host_ledger), 32 * sizeof(double)) != cudaSuccess) return bail(MPM_ERR_OUT_OF_MEMORY);
  const int ledger_blocks = h->num_sms * 4;
  if (cudaMalloc(reinterpret_cast<void**>(&h->ledger_partials), (ledger_blocks * 19 + 32) * sizeof(double)) != cudaSuccess)
    return bail(MPM_ERR_OUT_OF_MEMORY);
  h->ledger_out = h->ledger_partials + ledger_blocks * 19;
  // default material 0: fixed-corotated, unit moduli (the caller sets real materials)
  mpm_material def{};
  def.model = 0;
  def.mu = 1;
  def.lambda = 1;
  h->mats_host[0] = def;
  h->mats_dev[0] = mpm::material_to_device(def);
  if (alloc_grid(h) != MPM_OK) return bail(MPM_ERR_OUT_OF_MEMORY);
  mpm::g2p2g_blocks_per_sm(false);  // sets the dynamic shared memory limit of the no-scatter pass
  h->g2p2g_blocks = h->num_sms * mpm::g2p2g_blocks_per_sm(true);
  // The warp-specialised scatter passes (one 512-thread CTA per SM) are an autotuner candidate; on
  // the 2M-particle J2 drop they measured 0.49 ms per substep against 0.43 ms for the two-CTA
  // kernel, so they start off (MPM_B200_WS=1 makes them the default).
  const int ws_per_sm = mpm::ws_blocks_per_sm();
  h->ws_blocks = ws_per_sm > 0 ? h->num_sms * ws_per_sm : 0;
  h->ctx.ws_blocks = std::getenv("MPM_B200_WS") ? h->ws_blocks : 0;
  h->p2g_blocks = h->num_sms * mpm::p2g_blocks_per_sm();
  h->grid_blocks = h->num_sms * 8;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(MPM_ERR_CUDA);
  *out = h;
  return MPM_OK;
}

int mpm_destroy(mpm_handle* h) {
  if (!h) return MPM_ERR_INVALID_ARG;
  join_side(h);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->side) cudaStreamSynchronize(h->side);
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
  drop_graph(h);
  free_device(h);
  if (h->main_ev) cudaEventDestroy(h->main_ev);
  if (h->side_ev) cudaEventDestroy(h->side_ev);
  if (h->side) cudaStreamDestroy(h->side);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return MPM_OK;
}

const char* mpm_last_error(const mpm_handle* h) { return h ? h->err.c_str() : "null handle"; }

int mpm_configure_domain(mpm_handle* h, const mpm_domain* domain) {
  if (!h || !domain) return MPM_ERR_INVALID_ARG;
  SceneDev s;
  int rc = build_scene(h, *domain, s);
  if (rc != MPM_OK) return rc;
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  if (h->batch) return fail(h, MPM_ERR_STATE, "a batch handle's scenes are fixed at creation");
  h->dom = *domain;
  h->scene = s;
  h->scenes.assign(1, s);
  drop_graph(h);
  rc = alloc_grid(h);
  if (rc != MPM_OK) return rc;
  h->uploaded = false;  // positions are relative to the grid origin: upload again
  h->n = 0;
  return MPM_OK;
}

int mpm_grid_dims(const mpm_handle* h, int32_t dims[3], double origin[3]) {
  if (!h) return MPM_ERR_INVALID_ARG;
  for (int a = 0; a < 3; ++a) {
    if (dims) dims[a] = h->scene.dims[a];
    if (origin) origin[a] = h->scene.origin[a];
  }
  return MPM_OK;
}

int mpm_set_material(mpm_handle* h, int32_t index, const mpm_material* material) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (index < 0 || index >= kMaxMats) return fail(h, MPM_ERR_INVALID_ARG, "material index out of range [0, 256)");
  std::string why;
  const int rc = validate_material(material, why);
  if (rc != MPM_OK) return fail(h, rc, why);
  h->mats_host[index] = *material;
  h->mats_dev[index] = mpm::material_to_device(*material);
  h->mats_ext[index] = to_device_ext(*material);
  h->mat_set[index] = 1;
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<MaterialDev*>(h->ctx.mats) + index, &h->mats_dev[index], sizeof(MaterialDev),
                              cudaMemcpyHostToDevice, h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<mpm::MaterialExt*>(h->ctx.mats_ext) + index, &h->mats_ext[index],
                              sizeof(mpm::MaterialExt), cudaMemcpyHostToDevice, h->stream));
  refresh_flags(h);
  drop_graph(h);          // the kernel instances and the flags a captured graph holds may change
  h->grid_valid = false;  // stresses change
  h->last_estimate = 0;
  return MPM_OK;
}

int mpm_get_stream(mpm_handle* h, void** cuda_stream) {
  if (!h || !cuda_stream) return MPM_ERR_INVALID_ARG;
  *cuda_stream = h->stream;
  return MPM_OK;
}

static int ensure_staging(mpm_handle* h, size_t bytes) {
  if (h->staging_bytes >= bytes) return MPM_OK;
  if (h->staging) cudaFree(h->staging);
  h->staging = nullptr;
  h->staging_bytes = 0;
  MPM_CUDA(h, cudaMalloc(&h->staging, bytes));
  h->staging_bytes = bytes;
  return MPM_OK;
}

// Copies the caller's host arrays into device staging; fills ptrs with device addresses (or null).
// Staged arrays: 0-2 x, y, z; 3-5 v; 6 mass; 7 volume; 8 T; 9 plastic; 10 F; 11 C; 12 Jp; 13 dilation;
// 14 enthalpy.
constexpr int kStaged = 15;
static inline int staged_comps(int k) { return k == 10 || k == 11 ? 9 : 1; }

static int stage_in(mpm_handle* h, int64_t n, const mpm_particles* p, void* ptrs[kStaged], const int** mat_dev,
                    const unsigned char** pin_dev, unsigned fields, const unsigned char** melt_dev = nullptr) {
  const size_t es = p->dtype == MPM_F32 ? 4 : 8;
  const void* src[kStaged] = {p->x, p->y, p->z, p->vx, p->vy, p->vz, p->mass, p->volume, p->temperature, p->plastic,
                              p->F, p->C, p->jp, p->dilation, p->enthalpy};
  const unsigned need[kStaged] = {mpm::kFieldPos, mpm::kFieldPos, mpm::kFieldPos, mpm::kFieldVel, mpm::kFieldVel,
                                  mpm::kFieldVel, mpm::kFieldMass, mpm::kFieldVolume, mpm::kFieldTemp,
                                  mpm::kFieldPlastic, mpm::kFieldF, mpm::kFieldC, mpm::kFieldAux, mpm::kFieldAux,
                                  mpm::kFieldTemp};
  size_t total = 0;
  for (int k = 0; k < kStaged; ++k)
    if (src[k] && (fields & need[k])) total += align_up(staged_comps(k) * n * es, 256);
  if ((fields & mpm::kFieldMass) && p->material) total += align_up(n * 4, 256);
  if ((fields & mpm::kFieldMass) && p->pinned) total += align_up(n, 256);
  if ((fields & mpm::kFieldTemp) && p->melted && melt_dev) total += align_up(n, 256);
  int rc = ensure_staging(h, std::max<size_t>(total, 256));
  if (rc != MPM_OK) return rc;
  char* base = static_cast<char*>(h->staging);
  size_t off = 0;
  for (int k = 0; k < kStaged; ++k) {
    ptrs[k] = nullptr;
    if (!src[k] || !(fields & need[k])) continue;
    const size_t bytes = staged_comps(k) * n * es;
    ptrs[k] = base + off;
    MPM_CUDA(h, cudaMemcpyAsync(ptrs[k], src[k], bytes, cudaMemcpyHostToDevice, h->stream));
    off += align_up(bytes, 256);
  }
  *mat_dev = nullptr;
  *pin_dev = nullptr;
  if ((fields & mpm::kFieldMass) && p->material) {
    *mat_dev = reinterpret_cast<const int*>(base + off);
    MPM_CUDA(h, cudaMemcpyAsync(base + off, p->material, n * 4, cudaMemcpyHostToDevice, h->stream));
    off += align_up(n * 4, 256);
  }
  if ((fields & mpm::kFieldMass) && p->pinned) {
    *pin_dev = reinterpret_cast<const unsigned char*>(base + off);
    MPM_CUDA(h, cudaMemcpyAsync(base + off, p->pinned, n, cudaMemcpyHostToDevice, h->stream));
    off += align_up(n, 256);
  }
  if (melt_dev) *melt_dev = nullptr;
  if ((fields & mpm::kFieldTemp) && p->melted && melt_dev) {
    *melt_dev = reinterpret_cast<const unsigned char*>(base + off);
    MPM_CUDA(h, cudaMemcpyAsync(base + off, p->melted, n, cudaMemcpyHostToDevice, h->stream));
    off += align_up(n, 256);
  }
  MPM_CUDA(h, cudaMemcpyAsync(h->dptr_table, ptrs, kStaged * sizeof(void*), cudaMemcpyHostToDevice, h->stream));
  return MPM_OK;
}

int mpm_upload_particles(mpm_handle* h, int64_t n, const mpm_particles* p) {
  if (!h || !p || n < 0) return MPM_ERR_INVALID_ARG;
  if (n > h->cap) return fail(h, MPM_ERR_CAPACITY, "particle count exceeds the handle's capacity");
  if (p->dtype != MPM_F64 && p->dtype != MPM_F32) return fail(h, MPM_ERR_INVALID_ARG, "dtype must be MPM_F64 or MPM_F32");
  if (n > 0 && (!p->x || !p->y || !p->z || !p->mass || !p->volume))
    return fail(h, MPM_ERR_INVALID_ARG, "positions, mass and volume are required");
  bool single = true, pinned_any = false;
  if (h->batch) {
    // one material per scene, named at creation; particles come in scene order
    int64_t total = 0;
    for (size_t k = 0; k < h->scenes.size(); ++k) {
      total += h->scenes[k].p_end - h->scenes[k].p_begin;
      if (!h->mat_set[h->scene_material[k]]) return fail(h, MPM_ERR_INVALID_ARG, "a scene's material is not set");
    }
    if (n != total) return fail(h, MPM_ERR_INVALID_ARG, "a batch upload carries exactly the scenes' particle counts");
  } else if (p->material) {
    for (int64_t i = 0; i < n; ++i) {
      const int m = p->material[i];
      if (m < 0 || m >= kMaxMats || !h->mat_set[m]) return fail(h, MPM_ERR_INVALID_ARG, "particle material not set");
      if (m != p->material[0]) single = false;
    }
  } else if (!h->mat_set[0] && n > 0) {
    return fail(h, MPM_ERR_INVALID_ARG, "material 0 is not set");
  }
  if (p->pinned)
    for (int64_t i = 0; i < n && !pinned_any; ++i) pinned_any = p->pinned[i] != 0;
  const size_t es = p->dtype == MPM_F32 ? 4 : 8;
  if (n > 0 && p->dtype == MPM_F64) {
    const double* m = static_cast<const double*>(p->mass);
    const double* v = static_cast<const double*>(p->volume);
    for (int64_t i = 0; i < n; ++i)
      if (!(m[i] > 0) || !(v[i] > 0)) return fail(h, MPM_ERR_INVALID_ARG, "mass and volume must be positive");
  } else if (n > 0) {
    const float* m = static_cast<const float*>(p->mass);
    const float* v = static_cast<const float*>(p->volume);
    for (int64_t i = 0; i < n; ++i)
      if (!(m[i] > 0) || !(v[i] > 0)) return fail(h, MPM_ERR_INVALID_ARG, "mass and volume must be positive");
  }
  (void)es;
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  drop_graph(h);  // a captured graph holds the old particle count
  void* ptrs[kStaged];
  const int* mat_dev;
  const unsigned char* pin_dev;
  const unsigned char* melt_dev;
  const unsigned all = 0x1ffu;
  int rc = stage_in(h, n, p, ptrs, &mat_dev, &pin_dev, all, &melt_dev);
  if (rc != MPM_OK) return rc;
  h->ctx.n = n;
  h->ctx.has_pinned = pinned_any ? 1 : 0;
  h->ctx.single_material = single ? 1 : 0;
  if (p->temperature) h->ctx.has_thermal = 1;
  refresh_flags(h);
  MPM_CUDA(h, cudaMemsetAsync(h->ctx.time_scene, 0, sizeof(double) * h->scenes.size(), h->stream));
  if (h->batch) {
    // scene table already on the device (alloc_grid); each particle takes its scene's material
    { ProfScope ps(h, -1);
      mpm::launch_upload_convert(h->ctx, h->stream, n, p->dtype, reinterpret_cast<const void* const*>(h->dptr_table),
                                 nullptr, pin_dev, all, false, melt_dev); }
    MPM_CUDA(h, cudaGetLastError());
    h->n = n;
    h->uploaded = true;
    h->last_estimate = 0;
    h->grid_valid = false;
    h->reorder_pending = true;
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    return MPM_OK;
  }
  h->scene.mat_base = (single && p->material && n > 0) ? p->material[0] : 0;
  h->scene.p_begin = 0;
  h->scene.p_end = n;
  h->scenes[0] = h->scene;
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<SceneDev*>(h->ctx.scenes), &h->scene, sizeof(SceneDev), cudaMemcpyHostToDevice,
                              h->stream));
  // the conversion kernel writes the material index relative to mat_base = 0
  SceneDev tmp = h->scene;
  tmp.mat_base = 0;
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<SceneDev*>(h->ctx.scenes), &tmp, sizeof(SceneDev), cudaMemcpyHostToDevice, h->stream));
  { ProfScope ps(h, -1);
    mpm::launch_upload_convert(h->ctx, h->stream, n, p->dtype, reinterpret_cast<const void* const*>(h->dptr_table), mat_dev,
                               pin_dev, all, false, melt_dev); }
  MPM_CUDA(h, cudaGetLastError());
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<SceneDev*>(h->ctx.scenes), &h->scene, sizeof(SceneDev), cudaMemcpyHostToDevice,
                              h->stream));
  h->n = n;
  h->uploaded = true;
  h->last_estimate = 0;
  h->grid_valid = false;
  h->reorder_pending = true;
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  return MPM_OK;
}

static unsigned download_fields(const mpm_particles* p) {
  unsigned f = 0;
  if (p->x && p->y && p->z) f |= mpm::kFieldPos;
  if (p->vx && p->vy && p->vz) f |= mpm::kFieldVel;
  if (p->mass) f |= mpm::kFieldMass;
  if (p->volume) f |= mpm::kFieldVolume;
  if (p->temperature) f |= mpm::kFieldTemp;
  if (p->plastic) f |= mpm::kFieldPlastic;
  if (p->F) f |= mpm::kFieldF;
  if (p->C) f |= mpm::kFieldC;
  if (p->jp || p->dilation) f |= mpm::kFieldAux;
  if (p->enthalpy || p->melted) f |= mpm::kFieldTemp;
  return f;
}

int mpm_download_particles(mpm_handle* h, const mpm_particles* p) {
  if (!h || !p) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  const int64_t n = h->n;
  if (n == 0) return MPM_OK;
  const size_t es = p->dtype == MPM_F32 ? 4 : 8;
  const unsigned fields = download_fields(p);
  void* dst[kStaged] = {p->x, p->y, p->z, p->vx, p->vy, p->vz, p->mass, p->volume, p->temperature, p->plastic,
                        p->F, p->C, p->jp, p->dilation, p->enthalpy};
  size_t total = 0;
  for (int k = 0; k < kStaged; ++k)
    if (dst[k]) total += align_up(staged_comps(k) * n * es, 256);
  if (p->melted) total += align_up(n, 256);
  int rc = ensure_staging(h, std::max<size_t>(total, 256));
  if (rc != MPM_OK) return rc;
  void* dev[kStaged];
  char* base = static_cast<char*>(h->staging);
  size_t off = 0;
  for (int k = 0; k < kStaged; ++k) {
    dev[k] = nullptr;
    if (!dst[k]) continue;
    dev[k] = base + off;
    off += align_up(staged_comps(k) * n * es, 256);
  }
  MPM_CUDA(h, cudaMemcpyAsync(h->dptr_table, dev, kStaged * sizeof(void*), cudaMemcpyHostToDevice, h->stream));
  { ProfScope ps(h, -1); mpm::launch_download_convert(h->ctx, h->stream, n, p->dtype, reinterpret_cast<void* const*>(h->dptr_table), fields); }
  MPM_CUDA(h, cudaGetLastError());
  for (int k = 0; k < kStaged; ++k)
    if (dst[k]) MPM_CUDA(h, cudaMemcpyAsync(dst[k], dev[k], staged_comps(k) * n * es, cudaMemcpyDeviceToHost, h->stream));
  if (p->melted) {  // molten flags by caller index (u8 in the staging tail)
    unsigned char* mdev = static_cast<unsigned char*>(h->staging) + off;
    MPM_CUDA(h, cudaMemsetAsync(mdev, 0, n, h->stream));
    { ProfScope ps(h, -1); mpm::launch_download_melted(h->ctx, h->stream, n, mdev); }
    MPM_CUDA(h, cudaMemcpyAsync(p->melted, mdev, n, cudaMemcpyDeviceToHost, h->stream));
  }
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  return MPM_OK;
}

int mpm_count(const mpm_handle* h, int64_t* n) {
  if (!h || !n) return MPM_ERR_INVALID_ARG;
  *n = h->n;
  return MPM_OK;
}

int mpm_reset_deformation(mpm_handle* h) {
  if (!h) return MPM_ERR_INVALID_ARG;
  const mpm::Particles& p = h->ctx.p;
  MPM_CUDA(h, cudaMemsetAsync(p.C, 0, sizeof(float) * 9 * p.cap, h->stream));
  MPM_CUDA(h, cudaMemsetAsync(p.D, 0, sizeof(float) * 9 * p.cap, h->stream));
  MPM_CUDA(h, cudaMemsetAsync(p.ep, 0, sizeof(float) * p.cap, h->stream));
  MPM_CUDA(h, cudaMemsetAsync(p.aux, 0, sizeof(float) * p.cap, h->stream));  // Jp = 1, dilation = 0
  h->grid_valid = false;
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  return MPM_OK;
}

int mpm_stable_dt(mpm_handle* h, double* dt) {
  if (!h || !dt) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (h->n == 0) {
    *dt = h->scene.dt_max;
    return MPM_OK;
  }
  if (!h->grid_valid) {
    int rc = prepare_grid(h);
    if (rc != MPM_OK) return rc;
  }
  unsigned wg[2];
  MPM_CUDA(h, cudaMemcpyAsync(&wg[0], h->ctx.wave_max, 4, cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(&wg[1], h->ctx.grad_max, 4, cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  float wave, grad;
  std::memcpy(&wave, &wg[0], 4);
  std::memcpy(&grad, &wg[1], 4);
  const SceneDev& s = h->scene;
  *dt = std::min<double>(s.dt_max, std::min<double>(s.cfl * s.H / std::max(1.f, wave), s.grad_limit / std::max(1.f, grad)));
  return MPM_OK;
}

// Lays out the regularisation scratch for the current scenes and spacing: neighbour cells two
// spacings wide over each scene's grid, the cell sort and the per-particle shifts.
static int ensure_regularizer(mpm_handle* h) {
  if (!h->reg_dirty && h->rblock) return MPM_OK;
  const double hc = 2 * h->reg.spacing;
  const int ns = static_cast<int>(h->scenes.size());
  std::vector<mpm::RegScene> rs(ns);
  long long cells = 0;
  for (int s = 0; s < ns; ++s) {
    const SceneDev& sc = h->scenes[s];
    long long k = 1;
    for (int a = 0; a < 3; ++a) {
      const double ext = (sc.dims[a] - 1) * static_cast<double>(sc.H);
      rs[s].nc[a] = static_cast<int>(std::min(1.0e9, std::floor(ext / hc))) + 1;
      k *= rs[s].nc[a];
    }
    rs[s].cell_base = cells;
    cells += k;
    if (cells > (1ll << 30)) return fail(h, MPM_ERR_INVALID_ARG, "regularisation spacing too small for the grid");
  }
  const int64_t cap = h->cap;
  const size_t nb = mpm::reg_scan_blocks(cells);
  auto lay = [&](char* base, mpm::RegBufs& b, mpm::RegScene** scenes) {
    Carver cv{base};
    *scenes = cv.take<mpm::RegScene>(ns);
    b.count = cv.take<unsigned>(cells);
    b.start = cv.take<unsigned>(cells);
    b.cursor = cv.take<unsigned>(cells);
    b.block_sums = cv.take<unsigned>(nb + 1);
    b.largest = cv.take<unsigned>(ns);
    b.cell_of = cv.take<unsigned>(cap);
    b.sorted = cv.take<unsigned>(cap);
    b.target = cv.take<float>(cap);
    b.inv_mass = cv.take<float>(cap);
    b.shift = cv.take<float4>(cap);
    b.pos_sorted = cv.take<uint4>(cap);
    b.inv_sorted = cv.take<uint2>(cap);
    b.mat_sorted = cv.take<unsigned short>(cap);
    return align_up(cv.off, 256);
  };
  mpm::RegBufs probe{};
  mpm::RegScene* sp = nullptr;
  const size_t bytes = lay(nullptr, probe, &sp);
  if (h->rblock) cudaFree(h->rblock);
  h->rblock = nullptr;
  if (cudaMalloc(&h->rblock, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(h, MPM_ERR_OUT_OF_MEMORY, "regularisation scratch");
  }
  h->rblock_bytes = bytes;
  lay(static_cast<char*>(h->rblock), h->rbufs, &sp);
  MPM_CUDA(h, cudaMemcpyAsync(sp, rs.data(), sizeof(mpm::RegScene) * ns, cudaMemcpyHostToDevice, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));  // rs is a host temporary
  mpm::RegDev& r = h->rdev;
  r.scenes = sp;
  r.cells = cells;
  r.spacing = static_cast<float>(h->reg.spacing);
  r.inv_volume_unit = static_cast<float>(1.0 / h->reg.volume_unit);
  r.max_speed = static_cast<float>(h->reg.max_speed);
  r.rate = static_cast<float>(h->reg.rate);
  r.eps = static_cast<float>(h->reg.spacing * 1e-8 / 2.8);  // 1e-8 in the reference's units (spacing 2.8)
  r.inv_hc = static_cast<float>(1.0 / hc);
  h->reg_dirty = false;
  return MPM_OK;
}

// One regularisation pass over the current state; dt_scene (device, per scene) or dt.
static int regularize_now(mpm_handle* h, const float* dt_scene, double dt) {
  int rc = ensure_regularizer(h);
  if (rc != MPM_OK) return rc;
  mpm::RegDev r = h->rdev;
  r.dt_scene = dt_scene;
  r.dt = static_cast<float>(dt);
  h->ctx.n = h->n;
  { ProfScope ps(h, -1); mpm::launch_regularize(h->ctx, r, h->rbufs, h->stream); }
  MPM_CUDA(h, cudaGetLastError());
  h->grid_valid = false;  // positions moved: the next scatter re-sorts
  return MPM_OK;
}

// Substeps with the regularisation after each one (Simulation3.substep): a gather-only pass, the
// regularisation at the substep's dt, then the sort and scatter of the regularised state. The
// host reads the control block after each substep to stop when the call is done.
static int run_substeps_regularized(mpm_handle* h, int mode, double dt_req, int max_substeps, float dt_fixed,
                                    int* substeps, double* advanced) {
  if (!h->grid_valid) {
    int rc = prepare_grid(h);
    if (rc != MPM_OK) return rc;
  }
  h->ctx.n = h->n;
  { ProfScope ps(h, -1); mpm::launch_control_step(h->ctx, h->stream, mode, dt_req, max_substeps, dt_fixed); }
  for (int i = 0; i < max_substeps; ++i) {
    launch_substep(h, false);
    MPM_CUDA(h, cudaGetLastError());
    MPM_CUDA(h, cudaMemcpyAsync(h->host_ctrl, h->ctx.ctrl, sizeof(mpm::Ctrl), cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    const mpm::Ctrl ct = *h->host_ctrl;
    if (ct.done || (ct.status & (MPM_STATUS_NONFINITE | MPM_STATUS_TIMEOUT))) break;  // nothing ran
    h->grid_valid = false;
    h->pending_grid = false;  // the grid update consumed the scatter; the gather pass made none
    int rc = regularize_now(h, h->ctx.dt_scene, 0.0);
    if (rc != MPM_OK) return rc;
    if (h->reorder_interval > 0 && ++h->substeps_since_reorder >= h->reorder_interval) {
      h->reorder_pending = true;
      h->substeps_since_reorder = 0;
    }
    rc = prepare_grid(h);  // keeps the call's counters; clears only the lists and the done flag
    if (rc != MPM_OK) return rc;
    if (ct.substeps >= max_substeps || (mode == mpm::kModeRequested && !(ct.remaining > 1e-6 * dt_req))) break;
  }
  const mpm::Ctrl& ct = *h->host_ctrl;
  if (substeps) *substeps = ct.substeps;
  if (advanced) *advanced = ct.advanced;
  h->last_estimate = ct.substeps;
  return check_status(h);
}

// final_gather: the caller replaces the particle state after the call (mpm_frame_host), so the
// estimated last substep runs the gather-only pass; the scatter it would make is never used. If
// more substeps turn out to be needed, the state is scattered again (prepare_grid) first.
// nsteps (requested mode): requested-dt steps in this call, each of up to max_substeps substeps,
// with the step boundaries taken on the device (mpm_run).
static int run_substeps(mpm_handle* h, int mode, double dt_req, int max_substeps, float dt_fixed, int* substeps,
                        double* advanced, bool final_gather = false, int nsteps = 1) {
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (h->n == 0) {
    if (substeps) *substeps = 0;
    if (advanced) *advanced = 0;
    return MPM_OK;
  }
  if (h->reg.enabled) return run_substeps_regularized(h, mode, dt_req, max_substeps, dt_fixed, substeps, advanced);
  if (!h->grid_valid) {
    int rc = prepare_grid(h);
    if (rc != MPM_OK) return rc;
  }
  h->ctx.n = h->n;
  if (mode != mpm::kModeRequested) nsteps = 1;
  { ProfScope ps(h, -1); mpm::launch_control_step(h->ctx, h->stream, mode, dt_req, max_substeps, dt_fixed, nsteps); }
  // launches are bounded by max_substeps per requested step
  const long long max_total = static_cast<long long>(max_substeps) * nsteps;
  long long launched = 0;
  long long est;
  if (mode == mpm::kModeRequested && h->last_estimate > 0 && h->last_dt_requested == dt_req) {
    // the previous call's substep count per step for the same requested dt: no host round trip
    // before the launches (substeps past the end return at once; a short estimate is topped up)
    est = static_cast<long long>(std::min(h->last_estimate, max_substeps)) * nsteps;
  } else if (mode == mpm::kModeRequested) {
    double dt = 0;
    int rc = mpm_stable_dt(h, &dt);
    if (rc != MPM_OK) return rc;
    est = static_cast<long long>(std::ceil(dt_req / std::max(dt, 1e-30) - 1e-9));
    est = std::max(1ll, std::min(est, static_cast<long long>(max_substeps))) * nsteps;
  } else {
    est = max_substeps;
  }
  while (true) {
    for (long long i = 0; i < est; ++i) {
      launch_substep(h, !(final_gather && i == est - 1));
      // keep tiles contiguous in memory: a permutation pass after every reorder_interval substeps
      if (h->reorder_interval > 0 && ++h->substeps_since_reorder >= h->reorder_interval) {
        ProfScope ps(h, -1);
        const int rc = permute_state(h);
        if (rc != MPM_OK) return rc;
      }
    }
    launched += est;
    join_side(h);
    MPM_CUDA(h, cudaGetLastError());
    MPM_CUDA(h, cudaMemcpyAsync(h->host_ctrl, h->ctx.ctrl, sizeof(mpm::Ctrl), cudaMemcpyDeviceToHost, h->stream));
    MPM_CUDA(h, cudaStreamSynchronize(h->stream));
    const mpm::Ctrl& ct = *h->host_ctrl;
    const bool finished =
        ct.done || launched >= max_total ||
        (mode == mpm::kModeRequested
             ? ct.steps_left <= 1 && (!(ct.remaining > 1e-6 * dt_req) || ct.step_substeps >= max_substeps)
             : ct.substeps >= max_substeps);
    if (finished || (ct.status & (MPM_STATUS_NONFINITE | MPM_STATUS_TIMEOUT))) break;
    if (final_gather) {  // the last substep ran and made no scatter: scatter the state again
      h->pending_grid = false;
      const int rc = prepare_grid(h);
      if (rc != MPM_OK) return rc;
    }
    // the substeps still needed at this call's mean dt so far: the rest of the current step and
    // the steps not yet started
    est = 1;
    if (mode == mpm::kModeRequested && ct.substeps > 0 && ct.advanced > 0) {
      const double mean = ct.advanced / ct.substeps;
      const double need = std::ceil(ct.remaining / mean - 1e-9) + (ct.steps_left - 1) * std::ceil(dt_req / mean - 1e-9);
      est = static_cast<long long>(std::max(1.0, std::min(need, static_cast<double>(max_total - launched))));
    }
  }
  const mpm::Ctrl& ct = *h->host_ctrl;
  h->pending_grid = true;
  if (final_gather) {
    // every launch of the last batch ran (none returned at the done flag): the last one was the
    // gather-only pass and left no scatter; otherwise an earlier scatter pass was the last to run
    h->grid_valid = false;
    h->pending_grid = ct.substeps < launched;
  }
  if (substeps) *substeps = ct.substeps;
  if (advanced) *advanced = ct.advanced;
  h->last_estimate = mode == mpm::kModeRequested ? (ct.substeps + nsteps - 1) / nsteps : 0;
  h->last_dt_requested = dt_req;
  return status_error(h, ct.status);  // the control block was read after the last launch
}

int mpm_run(mpm_handle* h, double dt_requested, int32_t nsteps, int32_t max_substeps, int32_t* substeps,
            double* advanced) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!(dt_requested > 0) || !std::isfinite(dt_requested)) return fail(h, MPM_ERR_INVALID_ARG, "dt must be positive");
  if (nsteps <= 0) return fail(h, MPM_ERR_INVALID_ARG, "nsteps must be positive");
  if (max_substeps <= 0) max_substeps = 48;  // the reference's cap per step (src/three/simulation.js:308)
  // the call's substep counters (device control block, the returned count) are 32-bit
  if (static_cast<long long>(nsteps) * max_substeps > 0x7fffffffll)
    return fail(h, MPM_ERR_INVALID_ARG, "nsteps x max_substeps must stay below 2^31");
  if (h->reg.enabled) {  // the regulariser runs between substeps on the host's schedule: step by step
    int total = 0;
    double adv = 0;
    for (int k = 0; k < nsteps; ++k) {
      int sub = 0;
      double a = 0;
      const int rc = run_substeps(h, mpm::kModeRequested, dt_requested, max_substeps, 0.f, &sub, &a);
      if (rc != MPM_OK) return rc;
      total += sub;
      adv += a;
    }
    if (substeps) *substeps = total;
    if (advanced) *advanced = adv;
    return MPM_OK;
  }
  int sub = 0;
  const int rc = run_substeps(h, mpm::kModeRequested, dt_requested, max_substeps, 0.f, &sub, advanced, false, nsteps);
  if (substeps) *substeps = sub;
  return rc;
}

int mpm_step(mpm_handle* h, double dt_requested, int32_t max_substeps, int32_t* substeps, double* advanced) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!(dt_requested > 0) || !std::isfinite(dt_requested)) return fail(h, MPM_ERR_INVALID_ARG, "dt must be positive");
  if (max_substeps <= 0) max_substeps = 48;  // the reference's cap (src/three/simulation.js:308)
  int sub = 0;
  const int rc = run_substeps(h, mpm::kModeRequested, dt_requested, max_substeps, 0.f, &sub, advanced);
  if (substeps) *substeps = sub;
  return rc;
}

int mpm_step_fixed(mpm_handle* h, double dt, int32_t nsteps) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!(dt > 0) || nsteps <= 0) return fail(h, MPM_ERR_INVALID_ARG, "dt and nsteps must be positive");
  return run_substeps(h, mpm::kModeFixed, 0.0, nsteps, static_cast<float>(dt), nullptr, nullptr);
}

int mpm_step_cfl(mpm_handle* h, int32_t nsteps, double* time_advanced) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (nsteps <= 0) return fail(h, MPM_ERR_INVALID_ARG, "nsteps must be positive");
  return run_substeps(h, mpm::kModeCfl, 0.0, nsteps, 0.f, nullptr, time_advanced);
}

int mpm_step_host(mpm_handle* h, const mpm_particles* io, double dt) {
  if (!h || !io) return MPM_ERR_INVALID_ARG;
  if (h->batch) return fail(h, MPM_ERR_STATE, "single-scene call on a batch handle");
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (!(dt > 0)) return fail(h, MPM_ERR_INVALID_ARG, "dt must be positive");
  if (!io->x || !io->y || !io->z || !io->vx || !io->vy || !io->vz)
    return fail(h, MPM_ERR_INVALID_ARG, "positions and velocities are required");
  const int64_t n = h->n;
  if (n == 0) return MPM_OK;
  void* ptrs[kStaged];
  const int* mat_dev;
  const unsigned char* pin_dev;
  const unsigned fields = mpm::kFieldPos | mpm::kFieldVel;
  int rc = stage_in(h, n, io, ptrs, &mat_dev, &pin_dev, fields);
  if (rc != MPM_OK) return rc;
  { ProfScope ps(h, -1);
    mpm::launch_upload_convert(h->ctx, h->stream, n, io->dtype, reinterpret_cast<const void* const*>(h->dptr_table), nullptr,
                               nullptr, fields, true); }
  MPM_CUDA(h, cudaGetLastError());
  rc = prepare_grid(h);
  if (rc != MPM_OK) return rc;
  { ProfScope ps(h, -1); mpm::launch_control_step(h->ctx, h->stream, mpm::kModeFixed, 0.0, 1, static_cast<float>(dt)); }
  launch_substep(h, false);
  MPM_CUDA(h, cudaGetLastError());
  h->grid_valid = false;
  h->pending_grid = false;
  // positions and velocities back to the caller's arrays
  mpm_particles out{};
  out.dtype = io->dtype;
  out.x = io->x; out.y = io->y; out.z = io->z;
  out.vx = io->vx; out.vy = io->vy; out.vz = io->vz;
  rc = mpm_download_particles(h, &out);
  if (rc != MPM_OK) return rc;
  return check_status(h);
}

int mpm_frame_host(mpm_handle* h, const mpm_particles* io, double dt_requested, int32_t max_substeps,
                   int32_t* substeps) {
  if (!h || !io) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (!io->x || !io->y || !io->z || !io->vx || !io->vy || !io->vz)
    return fail(h, MPM_ERR_INVALID_ARG, "positions and velocities are required");
  const int64_t n = h->n;
  if (n == 0) return MPM_OK;
  void* ptrs[kStaged];
  const int* mat_dev;
  const unsigned char* pin_dev;
  const unsigned fields = mpm::kFieldPos | mpm::kFieldVel;
  int rc = stage_in(h, n, io, ptrs, &mat_dev, &pin_dev, fields);
  if (rc != MPM_OK) return rc;
  { ProfScope ps(h, -1);
    mpm::launch_upload_convert(h->ctx, h->stream, n, io->dtype, reinterpret_cast<const void* const*>(h->dptr_table), nullptr,
                               nullptr, fields, true); }
  MPM_CUDA(h, cudaGetLastError());
  h->grid_valid = false;
  if (!(dt_requested > 0) || !std::isfinite(dt_requested)) return fail(h, MPM_ERR_INVALID_ARG, "dt must be positive");
  if (max_substeps <= 0) max_substeps = 48;  // the reference's cap (src/three/simulation.js:308)
  // the next frame replaces positions and velocities again: the last substep needs no scatter
  rc = run_substeps(h, mpm::kModeRequested, dt_requested, max_substeps, 0.f, substeps, nullptr, true);
  if (rc != MPM_OK) return rc;
  mpm_particles out{};
  out.dtype = io->dtype;
  out.x = io->x; out.y = io->y; out.z = io->z;
  out.vx = io->vx; out.vy = io->vy; out.vz = io->vz;
  return mpm_download_particles(h, &out);
}

int mpm_set_regularizer(mpm_handle* h, const mpm_regularizer* r) {
  if (!h || !r) return MPM_ERR_INVALID_ARG;
  if (r->enabled && (!(r->spacing > 0) || !(r->volume_unit > 0) || !(r->max_speed > 0) || !(r->rate >= 0) ||
                     !std::isfinite(r->spacing) || !std::isfinite(r->volume_unit) || !std::isfinite(r->max_speed) ||
                     !std::isfinite(r->rate)))
    return fail(h, MPM_ERR_INVALID_ARG, "regulariser needs spacing, volume_unit, max_speed > 0 and rate >= 0");
  if (r->enabled && r->spacing != h->reg.spacing) h->reg_dirty = true;
  h->reg = *r;
  drop_graph(h);  // a captured graph holds the fused (unregularised) substeps
  return MPM_OK;
}

int mpm_regularize(mpm_handle* h, double dt) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(h, MPM_ERR_INVALID_ARG, "dt must be positive");
  if (!h->reg.enabled || h->n == 0) return MPM_OK;  // solidAntiClump off: nothing moves
  const int rc = regularize_now(h, nullptr, dt);
  if (rc != MPM_OK) return rc;
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  return MPM_OK;
}

// Lays out the heat-exchange scratch for cells one radius wide over each scene's grid.
static int ensure_heat(mpm_handle* h, double radius) {
  if (h->hblock && h->heat_radius == radius) return MPM_OK;
  const int ns = static_cast<int>(h->scenes.size());
  std::vector<mpm::RegScene> rs(ns);
  long long cells = 0;
  for (int s = 0; s < ns; ++s) {
    const SceneDev& sc = h->scenes[s];
    long long k = 1;
    for (int a = 0; a < 3; ++a) {
      const double ext = (sc.dims[a] - 1) * static_cast<double>(sc.H);
      rs[s].nc[a] = static_cast<int>(std::min(1.0e9, std::floor(ext / radius))) + 1;
      k *= rs[s].nc[a];
    }
    rs[s].cell_base = cells;
    cells += k;
    if (cells > (1ll << 30)) return fail(h, MPM_ERR_INVALID_ARG, "heat-exchange radius too small for the grid");
  }
  const int64_t cap = h->cap;
  const size_t nb = mpm::reg_scan_blocks(cells);
  auto lay = [&](char* base, mpm::HeatBufs& b, mpm::RegScene** scenes) {
    Carver cv{base};
    *scenes = cv.take<mpm::RegScene>(ns);
    b.count = cv.take<unsigned>(cells);
    b.start = cv.take<unsigned>(cells);
    b.cursor = cv.take<unsigned>(cells);
    b.block_sums = cv.take<unsigned>(nb + 1);
    b.exchanged = cv.take<double>(1);
    b.cell_of = cv.take<unsigned>(cap);
    b.sorted = cv.take<unsigned>(cap);
    b.pos_sorted = cv.take<uint4>(cap);
    b.prop_sorted = cv.take<float2>(cap);
    b.budget = cv.take<float>(cap);
    return align_up(cv.off, 256);
  };
  mpm::HeatBufs probe{};
  mpm::RegScene* sp = nullptr;
  const size_t bytes = lay(nullptr, probe, &sp);
  if (h->hblock) cudaFree(h->hblock);
  h->hblock = nullptr;
  h->heat_radius = 0;
  if (cudaMalloc(&h->hblock, bytes) != cudaSuccess) {
    cudaGetLastError();
    return fail(h, MPM_ERR_OUT_OF_MEMORY, "heat-exchange scratch");
  }
  if (!h->host_exchanged && cudaMallocHost(&h->host_exchanged, sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return fail(h, MPM_ERR_OUT_OF_MEMORY, "heat-exchange readback");
  }
  h->hblock_bytes = bytes;
  lay(static_cast<char*>(h->hblock), h->hbufs, &sp);
  MPM_CUDA(h, cudaMemcpyAsync(sp, rs.data(), sizeof(mpm::RegScene) * ns, cudaMemcpyHostToDevice, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));  // rs is a host temporary
  h->hdev.scenes = sp;
  h->hdev.cells = cells;
  h->heat_radius = radius;
  return MPM_OK;
}

int mpm_exchange_heat(mpm_handle* h, const mpm_heat_exchange* x, double dt, double* exchanged) {
  if (!h || !x) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (!(x->radius > 0) || !std::isfinite(x->radius) || !(x->geometry >= 0) || !(x->heat_rate >= 0) ||
      !(dt >= 0) || !std::isfinite(dt) || !std::isfinite(x->ambient_T) || !(x->ambient_rate >= 0))
    return fail(h, MPM_ERR_INVALID_ARG, "heat exchange needs radius > 0, geometry, heat_rate, dt >= 0");
  if (exchanged) *exchanged = 0;
  if (h->n == 0) return MPM_OK;
  int rc = ensure_heat(h, x->radius);
  if (rc != MPM_OK) return rc;
  mpm::HeatDev hd = h->hdev;
  hd.inv_hc = static_cast<float>(1.0 / x->radius);
  hd.radius = static_cast<float>(x->radius);
  hd.eps = static_cast<float>(x->radius * 1.25e-7);  // 1e-6 of the reference's 8-unit radius
  hd.geom_rate = static_cast<float>(x->geometry * x->heat_rate);
  hd.dt = static_cast<float>(dt);
  hd.ambient = x->ambient ? 1 : 0;
  hd.ambient_T = static_cast<float>(x->ambient_T);
  hd.ambient_rate = static_cast<float>(x->ambient_rate);
  h->ctx.n = h->n;
  { ProfScope ps(h, -1); mpm::launch_exchange_heat(h->ctx, hd, h->hbufs, h->stream); }
  MPM_CUDA(h, cudaGetLastError());
  MPM_CUDA(h, cudaMemcpyAsync(h->host_exchanged, h->hbufs.exchanged, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  if (exchanged) *exchanged = *h->host_exchanged;
  h->grid_valid = false;   // temperatures and possibly deformation changed: the next step re-scatters
  return MPM_OK;
}

int mpm_regularize_host(mpm_handle* h, const mpm_particles* io, double dt) {
  if (!h || !io) return MPM_ERR_INVALID_ARG;
  if (h->batch) return fail(h, MPM_ERR_STATE, "single-scene call on a batch handle");
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (!io->x || !io->y || !io->z) return fail(h, MPM_ERR_INVALID_ARG, "positions are required");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(h, MPM_ERR_INVALID_ARG, "dt must be positive");
  if (!h->reg.enabled || h->n == 0) return MPM_OK;
  void* ptrs[kStaged];
  const int* mat_dev;
  const unsigned char* pin_dev;
  int rc = stage_in(h, h->n, io, ptrs, &mat_dev, &pin_dev, mpm::kFieldPos);
  if (rc != MPM_OK) return rc;
  { ProfScope ps(h, -1);
    mpm::launch_upload_convert(h->ctx, h->stream, h->n, io->dtype, reinterpret_cast<const void* const*>(h->dptr_table),
                               nullptr, nullptr, mpm::kFieldPos, true); }
  MPM_CUDA(h, cudaGetLastError());
  rc = regularize_now(h, nullptr, dt);
  if (rc != MPM_OK) return rc;
  mpm_particles out{};
  out.dtype = io->dtype;
  out.x = io->x; out.y = io->y; out.z = io->z;
  return mpm_download_particles(h, &out);
}

// Opens the given faces of every scene (bit 2 axis + side): no separating-slip wall, no sticky
// floor and no position clamp there, because the domain continues in another scene or rank.
static void open_faces(mpm_handle* h, SceneDev& s, int faces) {
  for (int a = 0; a < 3; ++a) {
    const unsigned qmax = static_cast<unsigned>((static_cast<long long>(s.dims[a]) - 1) << mpm::kFracBits);
    if (faces & (1 << (2 * a))) {
      s.wall_lo[a] = -1;
      s.qlo[a] = 0;
      if (a == 1) s.sticky = 0;
    }
    if (faces & (1 << (2 * a + 1))) {
      s.wall_hi[a] = 1 << 30;
      s.qhi[a] = qmax;
    }
  }
  (void)h;
}

int mpm_batch_set_slabs(mpm_handle* h, int32_t planes) {
  if (!h) return MPM_ERR_INVALID_ARG;
  const int ns = static_cast<int>(h->scenes.size());
  if (!h->batch || ns < 2) return fail(h, MPM_ERR_STATE, "slabs need a batch handle of two or more scenes");
  if (h->slab_planes) return fail(h, MPM_ERR_STATE, "slabs are already set");
  if (planes < 4) return fail(h, MPM_ERR_INVALID_ARG, "slabs share at least 4 node planes");
  for (int s = 0; s + 1 < ns; ++s) {
    const SceneDev& a = h->scenes[s];
    const SceneDev& b = h->scenes[s + 1];
    const double H = a.H;
    bool ok = a.H == b.H && a.dims[0] == b.dims[0] && a.dims[1] == b.dims[1] && planes * 2 <= a.dims[2] &&
              planes * 2 <= b.dims[2];
    for (int k = 0; k < 2 && ok; ++k) ok = std::fabs(a.origin[k] - b.origin[k]) <= 1e-9 * H;
    ok = ok && std::fabs(b.origin[2] - (a.origin[2] + (a.dims[2] - planes) * H)) <= 1e-6 * H;
    if (!ok)
      return fail(h, MPM_ERR_INVALID_ARG,
                  "consecutive scenes must be slabs of one grid along z that share the given node planes");
  }
  for (int s = 0; s < ns; ++s) open_faces(h, h->scenes[s], (s > 0 ? 1 << 4 : 0) | (s + 1 < ns ? 1 << 5 : 0));
  h->scene = h->scenes[0];
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<SceneDev*>(h->ctx.scenes), h->scenes.data(), sizeof(SceneDev) * ns,
                              cudaMemcpyHostToDevice, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->slab_planes = planes;
  h->ctx.uniform_dt = 1;
  drop_graph(h);
  h->grid_valid = false;
  return MPM_OK;
}

int mpm_set_open_faces(mpm_handle* h, int32_t faces) {
  if (!h || faces < 0 || faces > 63) return MPM_ERR_INVALID_ARG;
  if (h->batch) return fail(h, MPM_ERR_STATE, "single-scene call on a batch handle");
  open_faces(h, h->scene, faces);
  h->scenes[0] = h->scene;
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<SceneDev*>(h->ctx.scenes), &h->scene, sizeof(SceneDev), cudaMemcpyHostToDevice,
                              h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->grid_valid = false;
  return MPM_OK;
}

int mpm_prepare(mpm_handle* h) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (h->n == 0 || h->grid_valid) return MPM_OK;
  const int rc = prepare_grid(h);
  if (rc != MPM_OK) return rc;
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  return MPM_OK;
}

static int halo_check(mpm_handle* h, int side, int planes, const void* buf) {
  if (h->batch) return fail(h, MPM_ERR_STATE, "single-scene call on a batch handle");
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if ((side != 0 && side != 1) || planes < 1 || planes * 2 > h->scene.dims[2])
    return fail(h, MPM_ERR_INVALID_ARG, "side 0 or 1 and 1 <= planes <= half the z nodes");
  if (!buf || (reinterpret_cast<uintptr_t>(buf) & 15u)) return fail(h, MPM_ERR_INVALID_ARG, "buffer must be 16-byte aligned");
  if (!h->grid_valid) return fail(h, MPM_ERR_STATE, "no fresh scatter: call mpm_prepare or a step first");
  return MPM_OK;
}

int mpm_halo_bytes(const mpm_handle* h, int32_t planes, int64_t* bytes) {
  if (!h || !bytes || planes < 1) return MPM_ERR_INVALID_ARG;
  const long long per = (long long)h->scene.gdim[0] * h->scene.gdim[1] * planes;
  *bytes = per * (32 + (h->ctx.conduct ? 4 : 0));
  return MPM_OK;
}

int mpm_halo_export(mpm_handle* h, int32_t side, int32_t planes, void* device_buffer) {
  if (!h) return MPM_ERR_INVALID_ARG;
  int rc = halo_check(h, side, planes, device_buffer);
  if (rc != MPM_OK) return rc;
  { ProfScope ps(h, -1); mpm::launch_halo_export(h->ctx, h->stream, side, planes, static_cast<float*>(device_buffer)); }
  MPM_CUDA(h, cudaGetLastError());
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  return MPM_OK;
}

int mpm_halo_add(mpm_handle* h, int32_t side, int32_t planes, const void* device_buffer) {
  if (!h) return MPM_ERR_INVALID_ARG;
  int rc = halo_check(h, side, planes, device_buffer);
  if (rc != MPM_OK) return rc;
  { ProfScope ps(h, -1); mpm::launch_halo_add(h->ctx, h->stream, side, planes, static_cast<const float*>(device_buffer)); }
  MPM_CUDA(h, cudaGetLastError());
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  return MPM_OK;
}

int mpm_profile_enable(mpm_handle* h, int32_t on) {
  if (!h) return MPM_ERR_INVALID_ARG;
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->profiling = on != 0;
  h->ev_used.clear();
  h->ev_next = 0;
  return MPM_OK;
}

int mpm_profile_read(mpm_handle* h, double ms[MPM_PROFILE_KERNELS], int64_t launches[MPM_PROFILE_KERNELS]) {
  if (!h || !ms || !launches) return MPM_ERR_INVALID_ARG;
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->side));  // the sort kernels' events
  for (int k = 0; k < MPM_PROFILE_KERNELS; ++k) {
    ms[k] = 0;
    launches[k] = 0;
  }
  for (const auto& u : h->ev_used) {
    if (u.first < 0 || u.first >= MPM_PROFILE_KERNELS) continue;
    float t = 0;
    MPM_CUDA(h, cudaEventElapsedTime(&t, h->ev_pool[u.second], h->ev_pool[u.second + 1]));
    ms[u.first] += t;
    launches[u.first] += 1;
  }
  return MPM_OK;
}

int mpm_check_bounded_wait(mpm_handle* h, int64_t limit_cycles, int32_t* timed_out) {
  if (!h || !timed_out) return MPM_ERR_INVALID_ARG;
  if (limit_cycles <= 0 || limit_cycles > (1ll << 33))
    return fail(h, MPM_ERR_INVALID_ARG, "limit_cycles must be in (0, 2^33]");
  join_side(h);
  unsigned* dev = nullptr;
  MPM_CUDA(h, cudaMalloc(&dev, sizeof(unsigned)));
  unsigned host = 0;
  mpm::launch_wait_probe(h->stream, dev, limit_cycles);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&host, dev, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(dev);
  if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, cudaGetErrorString(e));
  *timed_out = static_cast<int32_t>(host);
  return MPM_OK;
}

int mpm_launch_count(mpm_handle* h, int64_t* count) {
  if (!h || !count) return MPM_ERR_INVALID_ARG;
  *count = h->launches;
  return MPM_OK;
}

int mpm_ledger_compute(mpm_handle* h, mpm_ledger* out) {
  if (!h || !out) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  std::memset(out, 0, sizeof *out);
  h->ctx.n = h->n;
  const int blocks = h->num_sms * 4;
  { ProfScope ps(h, -1); ProfScope ps2(h, -1); mpm::launch_ledger(h->ctx, h->stream, h->ledger_partials, blocks, h->ledger_out); }
  MPM_CUDA(h, cudaGetLastError());
  MPM_CUDA(h, cudaMemcpyAsync(h->host_ledger, h->ledger_out, 19 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(h->host_ctrl, h->ctx.ctrl, sizeof(mpm::Ctrl), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  const double* r = h->host_ledger;
  out->mass = r[0];
  out->kinetic = r[1];
  out->affine = r[2];
  out->potential = r[3];
  out->elastic = r[4];
  for (int a = 0; a < 3; ++a) {
    out->momentum[a] = r[5 + a];
    out->angular[a] = r[8 + a];
  }
  out->min_j = h->n ? r[13] : 1.0;
  out->max_j = h->n ? r[14] : 1.0;
  out->max_plastic = r[15];
  out->max_von_mises = r[16];
  out->nonfinite = static_cast<int64_t>(r[17]);
  out->invalid_j = static_cast<int64_t>(r[18]);
  out->count = h->n;
  out->plastic_work = h->host_ctrl->plastic_work;
  return MPM_OK;
}

int mpm_min_j(mpm_handle* h, double* out) {
  if (!out) return MPM_ERR_INVALID_ARG;
  mpm_ledger L;
  const int rc = mpm_ledger_compute(h, &L);
  if (rc == MPM_OK) *out = L.min_j;
  return rc;
}

int mpm_status(mpm_handle* h, uint32_t* flags) {
  if (!h || !flags) return MPM_ERR_INVALID_ARG;
  MPM_CUDA(h, cudaMemcpyAsync(h->host_ctrl, h->ctx.ctrl, sizeof(mpm::Ctrl), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  *flags = h->host_ctrl->status;
  return MPM_OK;
}

int mpm_clear_status(mpm_handle* h) {
  if (!h) return MPM_ERR_INVALID_ARG;
  MPM_CUDA(h, cudaMemsetAsync(&h->ctx.ctrl->status, 0, sizeof(unsigned), h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  return MPM_OK;
}

int mpm_grid_debug(mpm_handle* h, double dt, double* mass, double* momentum) {
  if (!h || !mass || !momentum) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (!h->grid_valid) {
    const int rc = prepare_grid(h);
    if (rc != MPM_OK) return rc;
  }
  const SceneDev& s = h->scene;
  const size_t nodes = (size_t)s.dims[0] * s.dims[1] * s.dims[2];
  double* dev = nullptr;
  MPM_CUDA(h, cudaMalloc(&dev, nodes * 4 * sizeof(double)));
  mpm::launch_grid_debug(h->ctx, h->stream, 0, static_cast<float>(dt), dev, dev + nodes);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(mass, dev, nodes * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(momentum, dev + nodes, nodes * 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(dev);
  if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, cudaGetErrorString(e));
  return MPM_OK;
}

int mpm_snapshot(mpm_handle* h) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!h->snap) MPM_CUDA(h, cudaMalloc(&h->snap, h->pblock_bytes));
  MPM_CUDA(h, cudaMemcpyAsync(h->snap, h->pblock, h->pblock_bytes, cudaMemcpyDeviceToDevice, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->snap_valid = true;
  h->snap_n = h->n;
  return MPM_OK;
}

int mpm_rollback(mpm_handle* h) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!h->snap_valid) return fail(h, MPM_ERR_STATE, "no snapshot taken");
  MPM_CUDA(h, cudaMemcpyAsync(h->pblock, h->snap, h->pblock_bytes, cudaMemcpyDeviceToDevice, h->stream));
  MPM_CUDA(h, cudaMemsetAsync(&h->ctx.ctrl->status, 0, sizeof(unsigned), h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  if (h->n != h->snap_n) drop_graph(h);
  h->n = h->snap_n;
  h->grid_valid = false;
  return MPM_OK;
}

struct CheckpointHeader {
  uint32_t magic, version;
  int64_t n;
  mpm_domain dom;
  int32_t has_pinned, single_material, has_thermal, has_plastic, mat_base, has_aux;
};

// Raw device state of the n live particles, array by array, after a header with the domain and
// the materials (so a load reproduces the state bit for bit).
int mpm_checkpoint_save(mpm_handle* h, const char* path) {
  if (!h || !path) return MPM_ERR_INVALID_ARG;
  if (h->batch) return fail(h, MPM_ERR_STATE, "single-scene call on a batch handle");
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  FILE* f = std::fopen(path, "wb");
  if (!f) return fail(h, MPM_ERR_INVALID_ARG, std::string("cannot open ") + path);
  CheckpointHeader hd{kCheckpointMagic, kCheckpointVersion, h->n, h->dom, h->ctx.has_pinned, h->ctx.single_material,
                      h->ctx.has_thermal, h->ctx.has_plastic, h->scene.mat_base, h->ctx.has_aux};
  bool ok = std::fwrite(&hd, sizeof hd, 1, f) == 1;
  ok = ok && std::fwrite(h->mat_set.data(), 1, kMaxMats, f) == (size_t)kMaxMats;
  ok = ok && std::fwrite(h->mats_host.data(), sizeof(mpm_material), kMaxMats, f) == (size_t)kMaxMats;
  const mpm::Particles& p = h->ctx.p;
  struct Arr { const void* d; size_t es; int comps; } arrs[] = {
      {p.qx, 4, 1}, {p.qy, 4, 1}, {p.qz, 4, 1}, {p.vx, 4, 1}, {p.vy, 4, 1}, {p.vz, 4, 1}, {p.C, 4, 9}, {p.D, 4, 9},
      {p.m, 4, 1}, {p.V, 4, 1}, {p.ep, 4, 1}, {p.T, 4, 1}, {p.aux, 4, 1}, {p.latent, 4, 1}, {p.melted, 1, 1},
      {p.mat, 2, 1}, {p.pinned, 1, 1}, {p.id, 4, 1}};
  std::vector<char> buf;
  cudaStreamSynchronize(h->stream);
  for (const Arr& a : arrs) {
    for (int comp = 0; comp < a.comps && ok; ++comp) {
      const size_t bytes = a.es * h->n;
      buf.resize(bytes + 1);
      const char* src = static_cast<const char*>(a.d) + comp * a.es * p.cap;
      if (bytes && cudaMemcpy(buf.data(), src, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) ok = false;
      ok = ok && (bytes == 0 || std::fwrite(buf.data(), 1, bytes, f) == bytes);
    }
  }
  std::fclose(f);
  return ok ? MPM_OK : fail(h, MPM_ERR_CUDA, "checkpoint write failed");
}

int mpm_checkpoint_load(mpm_handle* h, const char* path) {
  if (!h || !path) return MPM_ERR_INVALID_ARG;
  if (h->batch) return fail(h, MPM_ERR_STATE, "single-scene call on a batch handle");
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(h, MPM_ERR_INVALID_ARG, std::string("cannot open ") + path);
  CheckpointHeader hd;
  bool ok = std::fread(&hd, sizeof hd, 1, f) == 1 && hd.magic == kCheckpointMagic && hd.version == kCheckpointVersion;
  if (!ok) {
    std::fclose(f);
    return fail(h, MPM_ERR_INVALID_ARG, "not a checkpoint of this format");
  }
  if (hd.n > h->cap) {
    std::fclose(f);
    return fail(h, MPM_ERR_CAPACITY, "checkpoint holds more particles than the handle's capacity");
  }
  std::vector<char> set(kMaxMats);
  std::vector<mpm_material> mats(kMaxMats);
  ok = std::fread(set.data(), 1, kMaxMats, f) == (size_t)kMaxMats &&
       std::fread(mats.data(), sizeof(mpm_material), kMaxMats, f) == (size_t)kMaxMats;
  if (!ok) {
    std::fclose(f);
    return fail(h, MPM_ERR_INVALID_ARG, "truncated checkpoint");
  }
  int rc = mpm_configure_domain(h, &hd.dom);
  if (rc != MPM_OK) {
    std::fclose(f);
    return rc;
  }
  for (int i = 0; i < kMaxMats; ++i)
    if (set[i]) mpm_set_material(h, i, &mats[i]);
  const mpm::Particles& p = h->ctx.p;
  struct Arr { void* d; size_t es; int comps; } arrs[] = {
      {p.qx, 4, 1}, {p.qy, 4, 1}, {p.qz, 4, 1}, {p.vx, 4, 1}, {p.vy, 4, 1}, {p.vz, 4, 1}, {p.C, 4, 9}, {p.D, 4, 9},
      {p.m, 4, 1}, {p.V, 4, 1}, {p.ep, 4, 1}, {p.T, 4, 1}, {p.aux, 4, 1}, {p.latent, 4, 1}, {p.melted, 1, 1},
      {p.mat, 2, 1}, {p.pinned, 1, 1}, {p.id, 4, 1}};
  std::vector<char> buf;
  cudaStreamSynchronize(h->stream);
  for (const Arr& a : arrs) {
    for (int comp = 0; comp < a.comps && ok; ++comp) {
      const size_t bytes = a.es * hd.n;
      buf.resize(bytes + 1);
      ok = bytes == 0 || std::fread(buf.data(), 1, bytes, f) == bytes;
      char* dst = static_cast<char*>(a.d) + comp * a.es * p.cap;
      if (ok && bytes && cudaMemcpy(dst, buf.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
    }
  }
  std::fclose(f);
  if (!ok) return fail(h, MPM_ERR_INVALID_ARG, "truncated checkpoint");
  h->n = hd.n;
  h->ctx.n = hd.n;
  h->ctx.has_pinned = hd.has_pinned;
  h->ctx.single_material = hd.single_material;
  h->ctx.has_thermal = hd.has_thermal;
  h->ctx.has_plastic = hd.has_plastic;
  h->ctx.has_aux = hd.has_aux;
  apply_return_mode(h);
  h->scene.mat_base = hd.mat_base;
  h->scene.p_begin = 0;
  h->scene.p_end = hd.n;
  h->scenes[0] = h->scene;
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<SceneDev*>(h->ctx.scenes), &h->scene, sizeof(SceneDev), cudaMemcpyHostToDevice,
                              h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->uploaded = true;
  h->last_estimate = 0;
  h->grid_valid = false;
  return MPM_OK;
}

int mpm_host_alloc(size_t bytes, void** out) {
  if (!out || bytes == 0) return MPM_ERR_INVALID_ARG;
  return cudaMallocHost(out, bytes) == cudaSuccess ? MPM_OK : MPM_ERR_OUT_OF_MEMORY;
}

int mpm_host_free(void* p) { return cudaFreeHost(p) == cudaSuccess ? MPM_OK : MPM_ERR_CUDA; }

int mpm_return_map_batch(const mpm_material* material, int64_t n, const double* F_in, const double* ep, const double* T,
                         double dt, double* F_out, double* dep, double* tau) {
  if (material && mpm::aux_model(material->model)) return MPM_ERR_UNSUPPORTED;  // needs Jp / dilation in and out
  std::string why;
  int rc = validate_material(material, why);
  if (rc != MPM_OK) return rc;
  if (n < 0 || (n > 0 && (!F_in || !F_out || !dep || !tau))) return MPM_ERR_INVALID_ARG;
  if (n == 0) return MPM_OK;
  const MaterialDev md = mpm::material_to_device(*material);
  double* d = nullptr;
  const size_t bytes = (size_t)n * (9 + 1 + 1 + 9 + 1 + 9) * sizeof(double);
  if (cudaMalloc(&d, bytes) != cudaSuccess) return MPM_ERR_OUT_OF_MEMORY;
  double *dF = d, *dep_in = dF + 9 * n, *dT = dep_in + n, *dFo = dT + n, *ddep = dFo + 9 * n, *dtau = ddep + n;
  cudaError_t e = cudaMemcpy(dF, F_in, 9 * n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && ep) e = cudaMemcpy(dep_in, ep, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && T) e = cudaMemcpy(dT, T, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    mpm::launch_return_map_batch(md, n, dF, ep ? dep_in : nullptr, T ? dT : nullptr, static_cast<float>(dt), dFo, ddep, dtau,
                                 nullptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(F_out, dFo, 9 * n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(dep, ddep, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(tau, dtau, 9 * n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? MPM_OK : MPM_ERR_CUDA;
}

// ---- grid heat conduction ----

int mpm_set_return_mode(mpm_handle* h, int32_t mode, mpm_surrogate* s, double gate_tol, int32_t newton) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (mode == MPM_RETURN_EXACT) {
    h->return_mode = MPM_RETURN_EXACT;
    apply_return_mode(h);
    drop_graph(h);
    return MPM_OK;
  }
  const bool net = mode == MPM_RETURN_LEARNED_GATED;
  if (!(net && s) && mode != MPM_RETURN_NEWTON_GATED)
    return fail(h, MPM_ERR_INVALID_ARG, "mode must be exact, learned_gated with a network, or newton_gated");
  if (net && !mpm::learned_model(surr::surrogate_model(s)))
    return fail(h, MPM_ERR_UNSUPPORTED, "the learned return mode serves networks trained for Johnson-Cook (models 6, 7)");
  if (!(gate_tol > 0) || !(gate_tol < 1)) return fail(h, MPM_ERR_INVALID_ARG, "gate_tol must lie in (0, 1)");
  if (newton < 0 || newton > 8) return fail(h, MPM_ERR_INVALID_ARG, "newton must lie in [0, 8]");
  if (h->ctx.has_aux || h->ctx.conduct)
    return fail(h, MPM_ERR_UNSUPPORTED, "the gated return modes serve scenes without conduction and without snow, sand "
                                        "or pressure materials");
  // one device block: the network's BF16 weights and FP32 parameters (learned mode), then the counts
  const size_t wbytes = surr::weights_bytes();
  if (!h->mlp_block) {
    MPM_CUDA(h, cudaMalloc(&h->mlp_block, wbytes + surr::kParams * sizeof(float) + 16));
  }
  char* base = static_cast<char*>(h->mlp_block);
  float* params = reinterpret_cast<float*>(base + wbytes);
  unsigned* counts = reinterpret_cast<unsigned*>(params + surr::kParams);
  if (net) {
    const int rc = surr::export_weights(s, base, params, h->stream);
    if (rc != MPM_OK) return fail(h, rc, "copying the network's weights failed");
  }
  MPM_CUDA(h, cudaMemsetAsync(counts, 0, 16, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->ctx.mlp_w = base;
  h->ctx.mlp_params = params;
  h->ctx.gate_counts = counts;
  h->ctx.gate_tol = static_cast<float>(gate_tol);
  h->ctx.learned_newton = newton;
  h->return_mode = mode;
  apply_return_mode(h);
  drop_graph(h);
  return MPM_OK;
}

int mpm_gate_counts_read(mpm_handle* h, mpm_gate_counts* out, int32_t reset) {
  if (!h || !out) return MPM_ERR_INVALID_ARG;
  *out = mpm_gate_counts{};
  if (!h->mlp_block) return MPM_OK;
  unsigned* counts = h->ctx.gate_counts;
  unsigned hc[2] = {0, 0};
  join_side(h);
  MPM_CUDA(h, cudaMemcpyAsync(hc, counts, sizeof hc, cudaMemcpyDeviceToHost, h->stream));
  if (reset) MPM_CUDA(h, cudaMemsetAsync(counts, 0, sizeof hc, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  out->learned = hc[0];
  out->fallback = hc[1];
  return MPM_OK;
}

int mpm_set_conduction(mpm_handle* h, int32_t scene, double conductivity, double density, double specific_heat) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (scene < 0 || scene >= (int)h->scenes.size()) return fail(h, MPM_ERR_INVALID_ARG, "scene index out of range");
  if (!(conductivity >= 0) || !std::isfinite(conductivity))
    return fail(h, MPM_ERR_INVALID_ARG, "conductivity must be finite and >= 0");
  SceneDev& s = h->scenes[scene];
  if (conductivity > 0) {
    if (!(density > 0) || !(specific_heat > 0)) return fail(h, MPM_ERR_INVALID_ARG, "density and specific heat must be > 0");
    const double H = s.H;
    s.cond_G = static_cast<float>(conductivity * H);
    s.cond_inv_mfull = static_cast<float>(1.0 / (density * H * H * H));
    s.cond_inv_cp = static_cast<float>(1.0 / specific_heat);
    s.cond_dt_max = static_cast<float>(0.9 * density * specific_heat * H * H / (6.0 * conductivity));
  } else {
    s.cond_G = s.cond_inv_mfull = s.cond_inv_cp = 0.f;
    s.cond_dt_max = 0.f;
  }
  if (scene == 0) {
    // keep the single-scene copy (and its particle range) in step
    SceneDev s0 = s;
    s0.p_begin = h->scene.p_begin;
    s0.p_end = h->scene.p_end;
    s0.mat_base = h->scene.mat_base;
    h->scene = s0;
    s = s0;
  }
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<SceneDev*>(h->ctx.scenes) + scene, &s, sizeof(SceneDev), cudaMemcpyHostToDevice,
                              h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  int any = 0;
  for (const SceneDev& x : h->scenes) any |= x.cond_G > 0.f;
  h->ctx.conduct = any;
  if (any) h->ctx.has_thermal = 1;  // temperatures are read and written
  apply_return_mode(h);
  drop_graph(h);
  h->grid_valid = false;  // the next scatter carries the heat channel
  return MPM_OK;
}

// ---- viewer frame ----

int mpm_pack_frame(mpm_handle* h, int64_t preview_limit, float* data, int64_t max_rows, mpm_frame_info* info) {
  if (!h || !info || preview_limit <= 0 || max_rows < 0 || (max_rows > 0 && !data)) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  std::memset(info, 0, sizeof *info);
  const int64_t n = h->n;
  const int64_t stride = std::max<int64_t>(1, (n + preview_limit - 1) / preview_limit);
  const int64_t rows = (n + stride - 1) / stride;
  info->count = n;
  info->stride = stride;
  info->rows = rows;
  if (rows > max_rows) return fail(h, MPM_ERR_CAPACITY, "data holds fewer rows than the frame needs");
  mpm_ledger L;
  int rc = mpm_ledger_compute(h, &L);
  if (rc != MPM_OK) return rc;
  info->mass = L.mass;
  info->min_j = L.min_j;
  info->max_von_mises = L.max_von_mises;
  info->max_plastic = L.max_plastic;
  info->nonfinite = L.nonfinite;
  if (n == 0) return MPM_OK;
  const size_t data_bytes = align_up(rows * 8 * sizeof(float), 256);
  rc = ensure_staging(h, data_bytes + 256 + 256 * sizeof(unsigned));
  if (rc != MPM_OK) return rc;
  char* base = static_cast<char*>(h->staging);
  float* d_data = reinterpret_cast<float*>(base);
  double* d_energy = reinterpret_cast<double*>(base + data_bytes);
  unsigned* d_tkey = reinterpret_cast<unsigned*>(base + data_bytes + 8);
  unsigned* d_counts = reinterpret_cast<unsigned*>(base + data_bytes + 256);
  const unsigned tinit[2] = {0xffffffffu, 0u};
  MPM_CUDA(h, cudaMemsetAsync(d_energy, 0, 8, h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(d_tkey, tinit, sizeof tinit, cudaMemcpyHostToDevice, h->stream));
  MPM_CUDA(h, cudaMemsetAsync(d_counts, 0, 256 * sizeof(unsigned), h->stream));
  h->ctx.n = n;
  { ProfScope ps(h, -1); mpm::launch_pack_frame(h->ctx, h->stream, stride, d_data, d_energy, d_tkey, d_counts); }
  MPM_CUDA(h, cudaGetLastError());
  double energy = 0;
  unsigned tkey[2], counts[256];
  MPM_CUDA(h, cudaMemcpyAsync(data, d_data, rows * 8 * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(&energy, d_energy, 8, cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(tkey, d_tkey, sizeof tkey, cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(counts, d_counts, sizeof counts, cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  auto unkey = [](unsigned k) {
    const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &u, 4);
    return static_cast<double>(f);
  };
  info->thermal_energy = energy;
  info->min_T = unkey(tkey[0]);
  info->max_T = unkey(tkey[1]);
  for (int k = 0; k < 256; ++k) info->per_material[k] = counts[k];
  bool finite = L.nonfinite == 0 && std::isfinite(L.mass) && std::isfinite(energy) && std::isfinite(L.min_j);
  for (int64_t i = 0; i < rows * 8 && finite; ++i) finite = std::isfinite(data[i]);
  if (!finite) return fail(h, MPM_ERR_NONFINITE, "non-finite particle state in the frame");
  return MPM_OK;
}

// ---- per-particle edits (MPM3.resetParticle / MPM3.remove) ----

// Two spare words at the end of the ledger output block hold the slots found on the device.
static long long* slot_words(mpm_handle* h) { return reinterpret_cast<long long*>(h->ledger_out + 24); }

static int find_slots(mpm_handle* h, int64_t a, int64_t b, long long out[2]) {
  h->ctx.n = h->n;
  mpm::launch_find_ids(h->ctx, h->stream, static_cast<unsigned>(a), static_cast<unsigned>(b), slot_words(h));
  MPM_CUDA(h, cudaGetLastError());
  MPM_CUDA(h, cudaMemcpyAsync(h->host_ledger + 24, slot_words(h), 2 * sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(out, h->host_ledger + 24, 2 * sizeof(long long));
  return MPM_OK;
}

int mpm_reset_particle(mpm_handle* h, int64_t index) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (index < 0 || index >= h->n) return fail(h, MPM_ERR_OUT_OF_RANGE, "particle index out of range");
  long long slots[2];
  int rc = find_slots(h, index, index, slots);
  if (rc != MPM_OK) return rc;
  if (slots[0] < 0) return fail(h, MPM_ERR_STATE, "particle index has no home slot");
  mpm::launch_edit_particle(h->ctx, h->stream, 0, static_cast<unsigned>(index), slot_words(h));
  MPM_CUDA(h, cudaGetLastError());
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->grid_valid = false;  // the particle's stress changed
  return MPM_OK;
}

int mpm_remove_particle(mpm_handle* h, int64_t index, int64_t last) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (h->batch) return fail(h, MPM_ERR_STATE, "single-scene call on a batch handle");
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (last != h->n - 1) return fail(h, MPM_ERR_INVALID_ARG, "last must be the current count - 1");
  if (index < 0 || index > last) return fail(h, MPM_ERR_OUT_OF_RANGE, "particle index out of range");
  long long slots[2];
  int rc = find_slots(h, index, last, slots);
  if (rc != MPM_OK) return rc;
  if (slots[0] < 0 || slots[1] < 0) return fail(h, MPM_ERR_STATE, "particle index has no home slot");
  mpm::launch_edit_particle(h->ctx, h->stream, 1, static_cast<unsigned>(index), slot_words(h));
  MPM_CUDA(h, cudaGetLastError());
  drop_graph(h);
  h->n -= 1;
  h->ctx.n = h->n;
  h->scene.p_end = h->n;
  h->scenes[0] = h->scene;
  MPM_CUDA(h, cudaMemcpyAsync(const_cast<SceneDev*>(h->ctx.scenes), &h->scene, sizeof(SceneDev), cudaMemcpyHostToDevice,
                              h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->grid_valid = false;
  h->reorder_pending = true;
  return MPM_OK;
}

// ---- batched ensembles ----

int mpm_batch_create(const mpm_scene_desc* scenes, int32_t nscenes, mpm_handle** out) {
  if (!out || !scenes || nscenes <= 0 || nscenes > MPM_MAX_SCENES) return MPM_ERR_INVALID_ARG;
  *out = nullptr;
  int64_t total = 0;
  for (int k = 0; k < nscenes; ++k) {
    if (scenes[k].count < 0 || scenes[k].material < 0 || scenes[k].material >= kMaxMats) return MPM_ERR_INVALID_ARG;
    total += scenes[k].count;
  }
  if (total <= 0 || total > ((int64_t)1 << 31)) return MPM_ERR_INVALID_ARG;
  mpm_handle* h = nullptr;
  int rc = mpm_create(&scenes[0].domain, total, &h);
  if (rc != MPM_OK) return rc;
  std::vector<SceneDev> list(nscenes);
  int64_t begin = 0;
  for (int k = 0; k < nscenes; ++k) {
    rc = build_scene(h, scenes[k].domain, list[k]);
    if (rc != MPM_OK) {
      mpm_destroy(h);
      return rc;
    }
    list[k].p_begin = begin;
    list[k].p_end = begin + scenes[k].count;
    list[k].mat_base = scenes[k].material;
    begin += scenes[k].count;
    h->scene_material.push_back(scenes[k].material);
  }
  h->scenes = list;
  h->batch = true;
  h->ctx.scene_material = 1;  // each particle takes its scene's material
  h->dom = scenes[0].domain;
  rc = alloc_grid(h);
  if (rc == MPM_OK && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = MPM_ERR_CUDA;
  if (rc != MPM_OK) {
    mpm_destroy(h);
    return rc;
  }
  *out = h;
  return MPM_OK;
}

int mpm_batch_count(const mpm_handle* h, int32_t* nscenes) {
  if (!h || !nscenes) return MPM_ERR_INVALID_ARG;
  *nscenes = static_cast<int32_t>(h->scenes.size());
  return MPM_OK;
}

// Captures `count` substeps (with the re-sort passes the eager loop would run) into a graph. A
// graph spans 2 x reorder_interval substeps, so its two permutation passes bring the particle
// buffers back to the parity they had at capture and every replay sees the same pointers.
static int capture_graph(mpm_handle* h, int count) {
  drop_graph(h);
  const bool prof = h->profiling;
  h->profiling = false;
  const int64_t launches0 = h->launches;  // captured launches run on replay, not now
  join_side(h);  // the graph starts with nothing pending on the side stream
  MPM_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < count; ++i) {
    launch_substep(h, true);
    if (h->reorder_interval > 0 && ++h->substeps_since_reorder >= h->reorder_interval) {
      ProfScope ps(h, -1);
      permute_state(h);
    }
  }
  join_side(h);  // and ends with the side stream joined back
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  h->profiling = prof;
  h->launches_per_graph = h->launches - launches0;
  h->launches = launches0;
  if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    h->graph = nullptr;
    return fail(h, MPM_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  h->graph_substeps = count;
  return MPM_OK;
}

static int eager_substep(mpm_handle* h) {
  launch_substep(h, true);
  if (h->reorder_interval > 0 && ++h->substeps_since_reorder >= h->reorder_interval) {
    ProfScope ps(h, -1);
    return permute_state(h);
  }
  return MPM_OK;
}

int mpm_batch_run(mpm_handle* h, int32_t nsteps, int32_t use_graph) {
  if (!h) return MPM_ERR_INVALID_ARG;
  if (nsteps <= 0) return fail(h, MPM_ERR_INVALID_ARG, "nsteps must be positive");
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (h->n == 0) return MPM_OK;
  if (!use_graph || h->reorder_interval <= 0 || h->reg.enabled) return mpm_step_cfl(h, nsteps, nullptr);
  if (!h->grid_valid) {
    int rc = prepare_grid(h);
    if (rc != MPM_OK) return rc;
  }
  h->ctx.n = h->n;
  { ProfScope ps(h, -1); mpm::launch_control_step(h->ctx, h->stream, mpm::kModeCfl, 0.0, nsteps, 0.f); }
  const int chunk = 2 * h->reorder_interval;
  int left = nsteps;
  // eager substeps until the re-sort phase is 0, so every graph replay starts at the same phase
  while (left > 0 && h->substeps_since_reorder != 0) {
    const int rc = eager_substep(h);
    if (rc != MPM_OK) return rc;
    --left;
  }
  if (left >= chunk) {
    // a graph holds the pointers of the buffer parity it was captured with
    if (h->graph && (h->graph_substeps != chunk || h->ctx.p.qx != h->graph_parity)) drop_graph(h);
    if (!h->graph) {
      h->graph_parity = h->ctx.p.qx;
      const int rc = capture_graph(h, chunk);
      if (rc != MPM_OK) return rc;
    }
    join_side(h);
    while (left >= chunk) {
      MPM_CUDA(h, cudaGraphLaunch(h->graph, h->stream));
      h->launches += h->launches_per_graph;
      left -= chunk;
    }
  }
  for (; left > 0; --left) {
    const int rc = eager_substep(h);
    if (rc != MPM_OK) return rc;
  }
  join_side(h);
  MPM_CUDA(h, cudaGetLastError());
  h->pending_grid = true;
  return check_status(h);
}

int mpm_batch_times(mpm_handle* h, double* time, double* last_dt) {
  if (!h) return MPM_ERR_INVALID_ARG;
  const size_t ns = h->scenes.size();
  std::vector<float> dts(ns);
  if (time) MPM_CUDA(h, cudaMemcpyAsync(time, h->ctx.time_scene, ns * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaMemcpyAsync(dts.data(), h->ctx.dt_scene, ns * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  if (last_dt)
    for (size_t k = 0; k < ns; ++k) last_dt[k] = dts[k];
  return MPM_OK;
}

int mpm_batch_ledger(mpm_handle* h, int32_t scene, mpm_ledger* out) {
  if (!h || !out) return MPM_ERR_INVALID_ARG;
  if (scene < 0 || scene >= (int)h->scenes.size()) return fail(h, MPM_ERR_INVALID_ARG, "scene index out of range");
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  // the ledger kernel over this scene's home range: particle arrays offset to p_begin, one scene
  const SceneDev& sc = h->scenes[scene];
  const long long pb = sc.p_begin;
  Ctx c = h->ctx;
  mpm::Particles& p = c.p;
  p.qx += pb; p.qy += pb; p.qz += pb;
  p.vx += pb; p.vy += pb; p.vz += pb;
  p.C += pb; p.D += pb;
  for (int e = 0; e < 9; ++e) {
    p.Cc[e] += pb;
    p.Dc[e] += pb;
  }
  p.m += pb; p.V += pb; p.ep += pb; p.T += pb; p.aux += pb;
  p.mat += pb; p.pinned += pb; p.id += pb;
  c.n = sc.p_end - sc.p_begin;
  c.scenes = h->ctx.scenes + scene;
  c.nscenes = 1;
  std::memset(out, 0, sizeof *out);
  const int blocks = h->num_sms * 4;
  { ProfScope ps(h, -1); ProfScope ps2(h, -1); mpm::launch_ledger(c, h->stream, h->ledger_partials, blocks, h->ledger_out); }
  MPM_CUDA(h, cudaGetLastError());
  MPM_CUDA(h, cudaMemcpyAsync(h->host_ledger, h->ledger_out, 19 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  const double* r = h->host_ledger;
  out->mass = r[0];
  out->kinetic = r[1];
  out->affine = r[2];
  out->potential = r[3];
  out->elastic = r[4];
  for (int a = 0; a < 3; ++a) {
    out->momentum[a] = r[5 + a];
    out->angular[a] = r[8 + a];
  }
  out->min_j = c.n ? r[13] : 1.0;
  out->max_j = c.n ? r[14] : 1.0;
  out->max_plastic = r[15];
  out->max_von_mises = r[16];
  out->nonfinite = static_cast<int64_t>(r[17]);
  out->invalid_j = static_cast<int64_t>(r[18]);
  out->count = c.n;
  return MPM_OK;
}

int mpm_batch_grid_debug(mpm_handle* h, int32_t scene, double dt, double* mass, double* momentum) {
  if (!h || !mass || !momentum) return MPM_ERR_INVALID_ARG;
  if (scene < 0 || scene >= (int)h->scenes.size()) return fail(h, MPM_ERR_INVALID_ARG, "scene index out of range");
  if (!h->uploaded) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (!h->grid_valid) {
    const int rc = prepare_grid(h);
    if (rc != MPM_OK) return rc;
  }
  const SceneDev& s = h->scenes[scene];
  const size_t nodes = (size_t)s.dims[0] * s.dims[1] * s.dims[2];
  double* dev = nullptr;
  MPM_CUDA(h, cudaMalloc(&dev, nodes * 4 * sizeof(double)));
  mpm::launch_grid_debug(h->ctx, h->stream, scene, static_cast<float>(dt), dev, dev + nodes);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(mass, dev, nodes * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(momentum, dev + nodes, nodes * 3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(dev);
  if (e != cudaSuccess) return fail(h, MPM_ERR_CUDA, cudaGetErrorString(e));
  return MPM_OK;
}

// Times trial substeps of one schedule from the snapshot; returns ms per substep.
static int time_schedule(mpm_handle* h, int ws, int blocks, int interval, int tma, int trial, double* ms) {
  int rc = mpm_rollback(h);
  if (rc != MPM_OK) return rc;
  drop_graph(h);
  h->ctx.ws_blocks = ws ? h->ws_blocks : 0;
  h->g2p2g_blocks = blocks;
  h->reorder_interval = interval;
  h->substeps_since_reorder = 0;
  h->ctx.use_tma = (tma && h->ctx.tmaps) ? 1 : 0;
  rc = mpm_step_cfl(h, 2, nullptr);  // warm-up: prepares the grid
  if (rc != MPM_OK) return rc;
  cudaEvent_t e0, e1;
  MPM_CUDA(h, cudaEventCreate(&e0));
  MPM_CUDA(h, cudaEventCreate(&e1));
  cudaEventRecord(e0, h->stream);
  rc = mpm_step_cfl(h, trial, nullptr);
  cudaEventRecord(e1, h->stream);
  cudaEventSynchronize(e1);
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t / trial;
  return rc;
}

int mpm_batch_autotune(mpm_handle* h, int32_t trial_substeps, mpm_tuning* out) {
  if (!h || !out) return MPM_ERR_INVALID_ARG;
  if (!h->uploaded || h->n == 0) return fail(h, MPM_ERR_STATE, "no particles uploaded");
  if (trial_substeps <= 0) trial_substeps = 8;
  int rc = mpm_snapshot(h);
  if (rc != MPM_OK) return rc;
  // the trials advance the scenes' clocks too: keep them to restore afterwards
  std::vector<double> clocks(h->scenes.size());
  MPM_CUDA(h, cudaMemcpyAsync(clocks.data(), h->ctx.time_scene, clocks.size() * sizeof(double), cudaMemcpyDeviceToHost,
                              h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  const int def_blocks = h->g2p2g_blocks, def_interval = h->reorder_interval, def_tma = h->ctx.use_tma;
  const int def_ws = h->ctx.ws_blocks > 0 ? 1 : 0;
  const int max_per_sm = mpm::g2p2g_blocks_per_sm(true);
  struct Cand { int ws, per_sm, interval, tma; };
  std::vector<Cand> cands;
  for (int ws = (h->ws_blocks > 0 ? 1 : 0); ws >= 0; --ws)
    for (int per_sm = 1; per_sm <= (ws ? 1 : max_per_sm); ++per_sm)
      for (int interval : {8, 32, 128})
        for (int tma : {1, 0}) {
          if (tma && !h->ctx.tmaps) continue;
          cands.push_back({ws, ws ? def_blocks / h->num_sms : per_sm, interval, tma});
        }
  double def_ms = 0;
  Cand pick{def_ws, std::max(1, def_blocks / h->num_sms), def_interval, def_tma};
  rc = time_schedule(h, def_ws, def_blocks, def_interval, def_tma, trial_substeps, &def_ms);
  if (rc != MPM_OK) return rc;
  double best = def_ms;
  for (const Cand& c : cands) {
    double ms = 0;
    rc = time_schedule(h, c.ws, c.per_sm * h->num_sms, c.interval, c.tma, trial_substeps, &ms);
    if (rc != MPM_OK) return rc;
    if (ms < best) {
      best = ms;
      pick = c;
    }
  }
  rc = mpm_rollback(h);
  if (rc != MPM_OK) return rc;
  MPM_CUDA(h, cudaMemcpyAsync(h->ctx.time_scene, clocks.data(), clocks.size() * sizeof(double), cudaMemcpyHostToDevice,
                              h->stream));
  MPM_CUDA(h, cudaStreamSynchronize(h->stream));
  h->g2p2g_blocks = pick.per_sm * h->num_sms;
  h->reorder_interval = pick.interval;
  h->substeps_since_reorder = 0;
  h->ctx.use_tma = pick.tma;
  h->ctx.ws_blocks = pick.ws ? h->ws_blocks : 0;
  drop_graph(h);
  out->warp_specialised = pick.ws;
  out->blocks_per_sm = pick.ws ? h->ws_blocks / h->num_sms : pick.per_sm;
  out->reorder_interval = pick.interval;
  out->use_tma = pick.tma;
  out->trials = static_cast<int32_t>(cands.size()) + 1;
  out->ms_per_substep = best;
  out->ms_per_substep_default = def_ms;
  return MPM_OK;
}

}  // extern "C"
