// Internal device data layout of the MLS-MPM step (not part of the C ABI).
//
// HBM layout (structure of arrays, one array per component, all 4-byte aligned and coalesced):
//   particles  qx,qy,qz  u32 fixed-point position in cell units from the scene's grid origin
//                        (22 fractional bits: 2^-22 cell resolution, grids up to 1023 nodes/axis)
//              vx,vy,vz  f32 velocity (m/s)
//              C[9]      f32 APIC affine matrix (1/s)
//              D[9]      f32 F - I (centred deformation gradient)
//              m, V      f32 mass, reference volume (read-only in the step)
//              ep, T     f32 plastic strain, temperature
//              mat       u16 material index, pinned u8 (read only when the scene needs them)
//              id        u32 caller's index of the particle held in this slot
//              key       u32 particle-tile key for the next counting sort, perm u32 sorted->home
//   The particle arrays are double-buffered: a permutation pass rewrites the state in tile order
//   (home order = sort order) at upload and periodically, so tiles read contiguous memory.
//   grid       acc0[2]   float4 (m, px, py, pz)  scatter accumulators, ping-pong by substep
//              acc1[2]   float4 (fx, fy, fz, pinned mass)  stress force (dt-free) channel
//              vel       float4 (vx, vy, vz, m) updated grid velocity, TMA source of the gather
//              node order per scene ((z*gy)+y)*gx+x, gx,gy,gz multiples of 4 (storage dims)
//   tiles      particle tile = 4x4x4 stencil bases; node tile = 4x4x4 nodes
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "mpm_b200.h"
#include "mpm_math.h"

namespace mpm {

constexpr int kFracBits = 22;
constexpr float kFixedOne = 4194304.0f;        // 2^22
constexpr float kInvFixedOne = 2.384185791015625e-07f;
constexpr int kTile = 4;                         // tile edge (cells / nodes)
constexpr int kWinG = 6;                         // gather window edge (nodes)
constexpr int kWinS = 8;                         // scatter window edge (nodes)
constexpr int kWinSNodes = kWinS * kWinS * kWinS;
constexpr int kChannels = 8;                     // m, px, py, pz, fx, fy, fz, pinned mass
constexpr int kBlock = 256;                      // threads per CTA in the particle kernels
constexpr int kMaxScenes = 4096;
constexpr int kMaxMaterials = 4096;

enum StepMode : int { kModeFixed = 0, kModeRequested = 1, kModeCfl = 2 };

struct SceneDev {
  float H, invH;
  int dims[3];          // reference node counts per axis
  int gdim[3];          // storage dims (4 * tiles + 4)
  int tiles[3];         // particle tiles per axis
  int ntiles[3];        // node tiles per axis (gdim / 4)
  long long node_base;  // first node of this scene in the grid arrays
  int tile_base;        // first particle tile (global id)
  int node_tile_base;   // first node tile (global id)
  int wall_lo[3];       // node index <= wall_lo: within one cell of lower (reference q < lower + h)
  int wall_hi[3];       // node index >= wall_hi: within one cell of upper (q > upper - h)
  unsigned qlo[3], qhi[3];  // fixed-point clamp range of positions
  int clamp, sticky;
  float gravity[3];
  float mass_eps;
  float cfl, dt_max, grad_limit;
  int mat_base, nmat;
  long long p_begin, p_end;  // home particle range
  double origin[3];
  // grid heat conduction between face-neighbour nodes (off when cond_G == 0):
  // conductance k h dt min(1, min(m_i, m_j) / (rho h^3)), node heat capacity m cp
  float cond_G;          // k h (W/K)
  float cond_inv_mfull;  // 1 / (rho h^3)
  float cond_inv_cp;     // 1 / cp
  float cond_dt_max;     // explicit-diffusion limit 0.9 rho cp h^2 / (6 k)
};

struct Ctrl {
  double remaining;     // requested-mode time left in this call
  double dt_requested;
  double advanced;
  double plastic_work;  // accumulated heat from plastic work (J), FP64
  int substeps;         // substeps done in this call
  int max_substeps;
  int done;
  int mode;
  float dt_fixed;
  unsigned step_index;  // parity source: grid state lives in acc[(step_index) & 1] before a substep
  unsigned status;      // MPM_STATUS_* flags
  unsigned work_count[2];
  unsigned work_next;
  unsigned active_count[2];
  unsigned grid_next;
  unsigned scan_ticket;
  int steps_left;        // requested-dt steps of this call still to start after the current one, + 1
  int step_substeps;     // substeps of the current requested-dt step
  unsigned sort_list;    // work list the sort after a scatter pass appends to (written by that pass)
  unsigned sort_active;  // 1 if that pass ran (the sort and scan skip a pass that returned at done)
  unsigned last_substep; // 1 when the current substep is the call's last (set by k_begin): only then
                         // does the fused pass store particle velocities and APIC matrices, which no
                         // later substep of the call reads
};

struct Particles {
  unsigned *qx, *qy, *qz;
  float *vx, *vy, *vz;
  float* C;   // 9 component arrays, stride cap
  float* D;   // 9 component arrays, stride cap
  float* Cc[9];  // the same component arrays as separate pointers (32-bit indexing in kernels)
  float* Dc[9];
  float *m, *V, *ep, *T;
  float* aux;       // Jp - 1 (snow, pressure models) or the dilation (sand); 0 for the other laws
  float* latent;    // molten fraction of a phase-change material on its latent plateau (0..1)
  unsigned char* melted;  // 1 once a phase-change material has fully melted
  unsigned short* mat;
  unsigned char* pinned;
  unsigned* id;     // caller's index of the particle in this home slot
  unsigned* key;    // shared by both particle buffers
  unsigned* perm;   // shared by both particle buffers
  long long cap;
};

struct Grid {
  float4* acc0[2];
  float4* acc1[2];
  float* heat[2];        // sum w m T (conduction only)
  float* tnode;          // node temperature of the last grid update (conduction only)
  float* mnode;          // node mass of the last grid update (conduction only)
  unsigned* tile_epoch;  // step index of a node tile's last grid update (conduction only)
  float4* vel;           // (vx, vy, vz, m), or (vx, vy, vz, dT) after a conduction pass
  unsigned* tile_flag;   // per node tile
  unsigned* active[2];   // active node-tile lists
};

struct SortBufs {
  unsigned* count;      // per particle tile, total_tiles + 1
  unsigned* start;      // block-local exclusive scan, total_tiles + 1
  unsigned* block_off;  // exclusive scan of block sums
  unsigned* rank;       // block-local exclusive count of non-empty tiles before each tile
  unsigned* block_rank; // exclusive scan of the blocks' non-empty tile counts
  uint4* work[2];       // (tile, start, count, scene), non-empty tiles in tile-key order
};

struct Ctx {
  Particles p;
  Grid g;
  SortBufs s;
  const SceneDev* scenes;
  const MaterialDev* mats;
  const MaterialExt* mats_ext;  // the constants of snow, sand and the pressure laws, same rows
  Ctrl* ctrl;
  float* dt_scene;      // per scene
  unsigned* wave_max;   // per scene, float bits of max(|v| + c * stretch)
  unsigned* grad_max;   // per scene, float bits of max sum|C|
  double* time_scene;   // per scene, simulated time accumulated by substeps
  const void* tmaps;    // per scene CUtensorMap (64-byte aligned), or null
  long long n;
  int nscenes;
  int total_tiles;
  int total_node_tiles;
  int has_pinned;
  int single_material;
  int scene_material;   // every particle has its scene's material (batch handles): one row per tile
  int has_thermal;      // temperature array is read and written
  int has_plastic;      // plastic strain array is read and written
  int has_aux;          // aux array is read and written (a snow, sand or pressure material is set)
  int use_tma;
  int ws_blocks;        // > 0: the particle passes that scatter run warp-specialised on this many CTAs
  int conduct;          // a scene conducts heat on the grid: heat channel, conduction pass, dT gather
  int uniform_dt;       // every scene takes the smallest scene dt (slabs of one domain)
  // learned return mode (Johnson-Cook laws): the network's BF16 weights and FP32 parameters (the
  // handle's own copy), the gate's residual tolerance, the most Newton steps after the prediction,
  // and the counts of returns the gate accepted and sent to the exact map (2 unsigned)
  int learned;         // 0 exact, 1 the network's guess, 2 the guess from the initial flow stress
  int learned_newton;
  float gate_tol;
  const void* mlp_w;
  const float* mlp_params;
  unsigned* gate_counts;
};

// Johnson-Cook returns the learned mode serves (src/three/metal-plasticity.js:28-34)
__host__ __device__ inline bool learned_model(int model) { return model == 6 || model == 7; }

#ifdef __CUDACC__
// Scene of home particle slot i (scenes hold contiguous slot ranges in order).
__device__ __forceinline__ int find_scene_by_particle(const SceneDev* sc, int ns, long long i) {
  int lo = 0, hi = ns - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sc[mid].p_begin <= i) lo = mid; else hi = mid - 1;
  }
  return lo;
}
#endif

// Device constants of a material (mpm_api.cu)
MaterialDev material_to_device(const mpm_material& m);

// Launch wrappers (mpm_kernels.cu)
void launch_control_init(const Ctx& c, cudaStream_t st);
void launch_keys(const Ctx& c, cudaStream_t st);
void launch_scan(const Ctx& c, cudaStream_t st, bool initial);
void launch_wait_probe(cudaStream_t st, unsigned* out, long long limit);
void launch_sort_scatter(const Ctx& c, cudaStream_t st, bool initial);
void launch_p2g(const Ctx& c, cudaStream_t st, int grid_blocks);
void launch_control_step(const Ctx& c, cudaStream_t st, int mode, double dt_req, int max_substeps, float dt_fixed,
                         int nsteps = 1);
void launch_begin(const Ctx& c, cudaStream_t st);
void launch_grid_clear(const Ctx& c, cudaStream_t st, int grid_blocks);
void launch_grid_update(const Ctx& c, cudaStream_t st, int grid_blocks);
void launch_conduct(const Ctx& c, cudaStream_t st, int grid_blocks);
// Slab decomposition along z: consecutive scenes share `planes` node planes; after a scatter both
// copies of every shared node hold the sum (only in node tiles the scene has active).
void launch_halo_sum(const Ctx& c, cudaStream_t st, int planes);
// One scene's low (side 0) or high (side 1) `planes` node planes of the fresh scatter, to or from
// a device buffer: acc0 planes, acc1 planes, then heat planes when conducting.
void launch_halo_export(const Ctx& c, cudaStream_t st, int side, int planes, float* buf);
void launch_halo_add(const Ctx& c, cudaStream_t st, int side, int planes, const float* buf);
void launch_g2p2g(const Ctx& c, cudaStream_t st, int grid_blocks, bool scatter);
void launch_ledger(const Ctx& c, cudaStream_t st, double* partials, int blocks, double* out);
void launch_grid_debug(const Ctx& c, cudaStream_t st, int scene, float dt, double* mass, double* mom);
void launch_upload_convert(const Ctx& c, cudaStream_t st, long long n, int dtype, const void* const* src,
                           const int* material, const unsigned char* pinned, unsigned fields, bool by_id,
                           const unsigned char* melted = nullptr);
void launch_download_melted(const Ctx& c, cudaStream_t st, long long n, unsigned char* out);
void launch_download_convert(const Ctx& c, cudaStream_t st, long long n, int dtype, void* const* dst,
                             unsigned fields);
void launch_permute(const Ctx& c, const Particles& dst, cudaStream_t st);
// viewer frame: sampled rows (8 floats) and energy / temperature-range / per-material reductions
void launch_pack_frame(const Ctx& c, cudaStream_t st, long long stride, float* data, double* energy, unsigned* tkey,
                       unsigned* counts);
// home slots of caller indices a and b into slots[0..1] (-1 when absent)
void launch_find_ids(const Ctx& c, cudaStream_t st, unsigned a, unsigned b, long long* slots);
// op 0: reset the deformation of slots[0]; op 1: drop slots[0], slots[1] takes caller index a
void launch_edit_particle(const Ctx& c, cudaStream_t st, int op, unsigned a, const long long* slots);
void launch_return_map_batch(const MaterialDev& m, long long n, const double* F_in, const double* ep,
                             const double* T, float dt, double* F_out, double* dep, double* tau,
                             cudaStream_t st);
int g2p2g_blocks_per_sm(bool scatter);
int ws_blocks_per_sm();
int p2g_blocks_per_sm();

// field bits of the conversion kernels
enum Field : unsigned {
  kFieldPos = 1u << 0, kFieldVel = 1u << 1, kFieldMass = 1u << 2, kFieldVolume = 1u << 3,
  kFieldTemp = 1u << 4, kFieldPlastic = 1u << 5, kFieldF = 1u << 6, kFieldC = 1u << 7,
  kFieldAux = 1u << 8
};

}  // namespace mpm
