/*
 * mpm_b200 — C ABI of the B200-native explicit MLS-MPM solid step.
 *
 * This is the drop-in boundary for the reference's JavaScript step/state API of the 3D solid
 * path (src/three/mpm.js:7-136, class MPM3) and the 2D facade named by it
 * (src/solid-mpm.js:20-116, class SolidMPM). A Node N-API addon, ctypes or any C caller binds
 * these functions; no PyTorch or C++ types cross the boundary. Plain pointers and sizes only.
 *
 * Ownership (reference: the caller owns particle arrays, MPM3 owns F, C and the grid,
 * src/three/mpm.js:8-18): the library owns every device buffer behind an opaque handle.
 * Upload and download functions take caller-owned host pointers and counts.
 *
 * Errors: every function returns an int status (MPM_OK = 0, negative on failure); no exception
 * crosses the ABI. mpm_last_error() returns a text for the last failure on a handle.
 * Threading: one handle per thread; calls on one handle are serialised on its own CUDA stream.
 */
#ifndef MPM_B200_H
#define MPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_ABI_VERSION 3

/* status codes */
#define MPM_OK 0
#define MPM_ERR_INVALID_ARG (-1)   /* reference: thrown Error on invalid domain (src/three/discretization.js:5-10) */
#define MPM_ERR_OUT_OF_MEMORY (-2)
#define MPM_ERR_CUDA (-3)
#define MPM_ERR_NONFINITE (-4)     /* reference: RuntimeError on non-finite state (gpu/solver.py:1033-1034) */
#define MPM_ERR_INVALID_J (-5)     /* det F <= 0 (src/simulation/particle-health.js:24-27) */
#define MPM_ERR_OUT_OF_RANGE (-6)  /* a particle left the grid */
#define MPM_ERR_TIMEOUT (-7)       /* a bounded device wait gave up */
#define MPM_ERR_STATE (-8)         /* call out of order (e.g. step before upload) */
#define MPM_ERR_CAPACITY (-9)      /* more particles than the handle's capacity
                                      (reference: create returns false at capacity, src/three/simulation.js:36) */
#define MPM_ERR_UNSUPPORTED (-10)  /* material model not built */

/* device status flags (mpm_status) */
#define MPM_STATUS_NONFINITE 0x1u
#define MPM_STATUS_INVALID_J 0x2u
#define MPM_STATUS_OUT_OF_RANGE 0x4u
#define MPM_STATUS_TIMEOUT 0x8u
#define MPM_STATUS_SCATTER_OVERFLOW 0x10u /* particle moved more than one cell in a substep (handled) */
#define MPM_STATUS_SORT_MISMATCH 0x20u    /* tile keys and counts disagreed; the affected writes were skipped */

/* material models (src/three/constitutive.js:6-19 numbering) */
#define MPM_MODEL_FIXED_COROTATED 0
#define MPM_MODEL_NEO_HOOKEAN 1
#define MPM_MODEL_SNOW 2                /* clamped principal stretches, compaction hardening */
#define MPM_MODEL_SAND 3                /* non-cohesive Drucker-Prager with a dilation history */
#define MPM_MODEL_J2 4
#define MPM_MODEL_J2_HARDENING 5
#define MPM_MODEL_JOHNSON_COOK 6        /* rate- and temperature-dependent, bisection return */
#define MPM_MODEL_JOHNSON_COOK_SIMPLE 7 /* Johnson-Cook without thermal softening */
#define MPM_MODEL_THERMAL_J2 10
#define MPM_MODEL_COHESIVE_DP 8         /* cohesive Drucker-Prager: dilatancy, tension cutoff */
#define MPM_MODEL_FOAM 9                /* Deshpande-Fleck foam: pressure-dependent yield, bisection return */
#define MPM_MODEL_NORTON_CREEP 11       /* Arrhenius power-law creep, bisection return */

/* element type of the floating-point arrays of mpm_particles */
#define MPM_F64 0
#define MPM_F32 1

/* Grid and boundary description (src/three/discretization.js:3-15): origin is
 * floor(lower/h)*h - 2h, nodes per axis ceil((upper-origin)/h) + 3. Walls: separating slip on all
 * six faces (src/three/mpm.js:93); optional sticky floor (every velocity component zero within one
 * cell of lower[1]). CFL rule (src/three/mpm.js:43-55 in SI): dt <= min(dt_max,
 * cfl*h/max(1, |v| + c*max(1, |F|_row |F|_col, compression)), grad_limit/max(1, sum|C|)),
 * c = sqrt((lambda + 2 mu) V / m). */
typedef struct mpm_domain {
  double lower[3];
  double upper[3];
  double cell_size;
  double gravity[3];       /* applied on the grid: v += dt g (equivalent to the reference's
                              particle-side v += g dt before P2G, src/three/simulation.js:337-344) */
  int32_t sticky_floor;
  int32_t clamp_positions; /* clamp particles into [lower, upper] after advection
                              (src/three/simulation.js:358-365) */
  double mass_eps;         /* node mass threshold, 1e-12 in the reference (src/three/mpm.js:89) */
  double cfl;              /* 0.175 reproduces the reference's 1.4*(h/8) */
  double dt_max;           /* h/1920 in reference units; <= 0 means unbounded */
  double grad_limit;       /* 0.08 in the reference */
  int32_t cubic;           /* 1: every axis uses max(nodes) like src/three/mpm.js:18 */
  int32_t reserved;
} mpm_domain;

/* Material (SI). Reference units are mu = lambda = 0.4 E and strengths as stress / E
 * (src/three/mpm.js:34-37). J2: q = sqrt(6) mu |dev e| / J, yield A + B ep
 * (src/three/metal-plasticity.js:12-27); thermal J2: (A + B ep)(1 - (1 - hot_ratio) theta),
 * theta = clamp((T - T_ref)/(T_hot - T_ref), 0, 1) (src/three/thermal-plasticity.js:12-29). */
typedef struct mpm_material {
  int32_t model;
  int32_t reserved;
  double mu;
  double lambda;
  double yield_stress;   /* A */
  double hardening;      /* B (model 5) or H (model 10) */
  double T_ref;
  double T_hot;
  double hot_ratio;
  double heat_fraction;  /* beta: share of plastic work converted to heat (gpu/mixed_material.py:150-172) */
  double specific_heat;  /* cp, J/kg/K */
  /* Johnson-Cook, models 6 and 7 (src/three/metal-plasticity.js:3,12-19): flow stress
   * (A + B ep^n)(1 + C ln max(1, rate / rate0))(1 - theta^m), theta from T_ref to T_melt (model 6) */
  double jc_n, jc_C, jc_rate0, T_melt, jc_m;
  /* Norton creep, model 11 (src/three/thermal-plasticity.js:3,17-21): strain rate
   * rate exp(clamp(Q/R (1/(T_ref + off) - 1/(T + off)), -60, 60)) (q / stress)^n */
  double creep_rate, creep_Q, creep_n, creep_stress;
  double temperature_offset; /* off: 273.15 when temperatures are in deg C like the reference, 0 in K */
  /* Snow, model 2 (src/three/constitutive.js:48,58-60): principal stretches clamped to
   * [1 - yield_strain, 1 + 0.3 yield_strain], Jp = clamp(Jp det F / det F', 0.6, 20), moduli
   * scaled by clamp(exp(10 (1 - Jp)), 0.25, 4). Sand, model 3 (constitutive.js:66-74): friction
   * angle in degrees. The reference takes both per particle; here they are per material. */
  double yield_strain, friction_deg;
  /* Cohesive Drucker-Prager, model 8, and Deshpande-Fleck foam, model 9
   * (src/three/pressure-plasticity.js:2,11-48): strengths in Pa (Cauchy, tension positive). */
  double dp_cohesion, dp_slope, dp_dilatancy, dp_tension;
  double df_alpha, df_plateau, df_gamma, df_densify, df_beta, df_eps_d;
  /* Particle-pair heat exchange (src/thermal.js:35-56): conductivity k (W/m/K). Enthalpy phase
   * change of the custom MPM material (src/three/phase-change.js:4-18): enabled when
   * latent_heat > 0 (J/kg), melting at melting_point; h = specific_heat T (+ latent_heat once
   * molten), the temperature sits at melting_point on the plateau, and a particle switches phase
   * only at complete melting or freezing. */
  double conductivity, melting_point, latent_heat;
} mpm_material;

/* Host particle arrays (structure of arrays, like Simulation3's Float64Arrays,
 * src/three/simulation.js:27-30; F and C are n x 9 row-major like MPM3.F, src/three/mpm.js:9).
 * Any pointer may be NULL: on upload NULL means the default (v = 0, F = I, C = 0, ep = 0,
 * T = 0, material 0, not pinned, Jp = 1, dilation = 0); on download NULL arrays are skipped. */
typedef struct mpm_particles {
  int32_t dtype;         /* MPM_F64 or MPM_F32 for every floating-point array below */
  int32_t reserved;
  void* x; void* y; void* z;
  void* vx; void* vy; void* vz;
  void* mass;
  void* volume;
  void* temperature;
  void* plastic;         /* accumulated plastic strain (MPM3.plastic) */
  void* F;               /* n x 9 */
  void* C;               /* n x 9 */
  int32_t* material;     /* index into the materials set with mpm_set_material */
  uint8_t* pinned;       /* pinned particles scatter but are not moved (src/three/mpm.js:84,108) */
  void* jp;              /* plastic volume ratio MPM3.Jp (models 2, 8, 9; 1 otherwise) */
  void* dilation;        /* MPM3.dilation (model 3; 0 otherwise) */
  void* enthalpy;        /* Simulation3.enthalpy (J/kg); on upload it sets the temperature (and phase) */
  uint8_t* melted;       /* Simulation3.melted: 1 once a phase-change material has fully melted */
} mpm_particles;

/* FP64 ledger, reduced on the device (src/simulation/mechanical-diagnostics.js:16-37 and
 * src/simulation/particle-health.js:12-30, SI units). */
typedef struct mpm_ledger {
  double mass, kinetic, affine, potential, elastic;
  double momentum[3];
  double angular[3];     /* includes the APIC spin m (h^2/4) (C21-C12, C02-C20, C10-C01) */
  double min_j, max_j, max_plastic, max_von_mises;
  double plastic_work;   /* heat put into particles by plastic work so far (J) */
  int64_t count, nonfinite, invalid_j;
} mpm_ledger;

typedef struct mpm_handle mpm_handle;

/* ---- lifetime (new MPM3(capacity), configure(domain): src/three/mpm.js:8-19) ---- */
int mpm_abi_version(void);
const char* mpm_error_string(int status);
int mpm_create(const mpm_domain* domain, int64_t capacity, mpm_handle** out);
int mpm_destroy(mpm_handle* h);
const char* mpm_last_error(const mpm_handle* h);
int mpm_configure_domain(mpm_handle* h, const mpm_domain* domain);
int mpm_grid_dims(const mpm_handle* h, int32_t dims[3], double origin[3]);
int mpm_set_material(mpm_handle* h, int32_t index, const mpm_material* material);
/* The checks mpm_set_material applies, on the host without a handle (like the reference's
 * pressureParameters, src/three/pressure-plasticity.js:4-10): MPM_OK, MPM_ERR_INVALID_ARG or
 * MPM_ERR_UNSUPPORTED. */
int mpm_validate_material(const mpm_material* material);
int mpm_get_stream(mpm_handle* h, void** cuda_stream);

/* ---- state (Simulation3 arrays + MPM3.F/C/plastic) ---- */
int mpm_upload_particles(mpm_handle* h, int64_t n, const mpm_particles* p);
int mpm_download_particles(mpm_handle* h, const mpm_particles* p);
int mpm_count(const mpm_handle* h, int64_t* n);
/* MPM3.reset() / resetParticle for all: F = I, C = 0, plastic = 0 (src/three/mpm.js:20-21) */
int mpm_reset_deformation(mpm_handle* h);
/* MPM3.resetParticle(p) (src/three/mpm.js:21): F = I, C = 0, plastic = 0 for the caller's
 * particle index p (the index used at upload). */
int mpm_reset_particle(mpm_handle* h, int64_t index);
/* MPM3.remove(p, last) with the caller's Simulation3.remove(i) (src/three/mpm.js:22-25,
 * src/three/simulation.js:114): particle `last` takes index p with all of its state and the
 * count drops by one; `last` must be the current count - 1. Single-scene handles only. */
int mpm_remove_particle(mpm_handle* h, int64_t index, int64_t last);

/* ---- stepping ---- */
/* MPM3.stableStep(s) (src/three/mpm.js:40-55) on the current state */
int mpm_stable_dt(mpm_handle* h, double* dt);
/* Simulation3.step(dt) sub-stepping (src/three/simulation.js:305-311): advance by dt_requested in
 * substeps of min(remaining, stable dt), at most max_substeps; the state stays on the device. */
int mpm_step(mpm_handle* h, double dt_requested, int32_t max_substeps, int32_t* substeps,
             double* advanced);
/* nsteps consecutive mpm_step calls in one call: every requested-dt step sub-steps to the CFL
 * limit as mpm_step does (at most max_substeps each), the step boundaries are taken on the
 * device and the host synchronises once at the end. *substeps is the total over all steps,
 * *advanced the time advanced (nsteps x dt_requested unless a step hit max_substeps). */
int mpm_run(mpm_handle* h, double dt_requested, int32_t nsteps, int32_t max_substeps, int32_t* substeps,
            double* advanced);
/* nsteps substeps of exactly dt each (no CFL control) */
int mpm_step_fixed(mpm_handle* h, double dt, int32_t nsteps);
/* nsteps substeps, each of the scene's own stable dt (ensemble / CFL mode) */
int mpm_step_cfl(mpm_handle* h, int32_t nsteps, double* time_advanced);
/* MPM3.step(s, dt) drop-in (src/three/mpm.js:56-134): positions and velocities come from the
 * caller's host arrays, one step of dt runs, and positions and velocities are written back.
 * F, C and plastic strain stay on the device (MPM3 owns them). */
int mpm_step_host(mpm_handle* h, const mpm_particles* io, double dt);

/* Simulation3.step(dt) drop-in for the solid path (src/three/simulation.js:305-311): positions and
 * velocities come from the caller's host arrays, the step advances dt_requested in CFL substeps on
 * the device, and positions and velocities are written back. The call's last substep skips the
 * scatter that the next call's upload would replace, so a following mpm_step scatters the state
 * again first (same results, one extra scatter pass). */
int mpm_frame_host(mpm_handle* h, const mpm_particles* io, double dt_requested, int32_t max_substeps,
                   int32_t* substeps);

/* ---- diagnostics ---- */
int mpm_ledger_compute(mpm_handle* h, mpm_ledger* out);
/* MPM3.minJ(s) (src/three/mpm.js:135) */
int mpm_min_j(mpm_handle* h, double* out);
int mpm_status(mpm_handle* h, uint32_t* flags);
/* Self-check of the device's bounded waits (the TMA window waits of the particle pass give up
 * after about a second, set MPM_STATUS_TIMEOUT and leave the context usable): waits on a barrier
 * that nothing completes for limit_cycles SM cycles on the handle's stream and reports
 * *timed_out = 1 when the wait gave up. No other state changes. */
int mpm_check_bounded_wait(mpm_handle* h, int64_t limit_cycles, int32_t* timed_out);
int mpm_clear_status(mpm_handle* h);
/* Grid after P2G of the current state with a step of dt: node mass and momentum including
 * dt * (stress force + m g), in node order ((z*ny)+y)*nx+x. Arrays of nx*ny*nz and 3*nx*ny*nz. */
int mpm_grid_debug(mpm_handle* h, double dt, double* mass, double* momentum);

/* Per-kernel device time, measured with CUDA events on the handle's stream around each launch
 * while enabled (reference: s.profile stage timers, src/three/mpm.js:60-133).
 * Kernel ids: 0 begin, 1 grid update, 2 g2p2g, 3 scan, 4 sort scatter, 5 p2g, 6 keys. */
#define MPM_PROFILE_KERNELS 7
int mpm_profile_enable(mpm_handle* h, int32_t on);
int mpm_profile_read(mpm_handle* h, double ms[MPM_PROFILE_KERNELS], int64_t launches[MPM_PROFILE_KERNELS]);
/* number of kernels this handle has launched (all kinds) */
int mpm_launch_count(mpm_handle* h, int64_t* count);

/* ---- rollback and checkpoint (gpu/mixed_solver.py:453-480 keeps in-memory rollback copies) ---- */
int mpm_snapshot(mpm_handle* h);
int mpm_rollback(mpm_handle* h);
int mpm_checkpoint_save(mpm_handle* h, const char* path);
int mpm_checkpoint_load(mpm_handle* h, const char* path);

/* ---- pinned host memory for fast uploads ---- */
int mpm_host_alloc(size_t bytes, void** out);
int mpm_host_free(void* p);

/* ---- grid heat conduction ----
 * No counterpart in the reference's solid step (its particles exchange heat pairwise,
 * gpu/solver.py:775-811); this is the grid conduction of the coupled scene: each substep P2G
 * also scatters sum w m T, node temperatures T_i follow, face-neighbour nodes that both hold
 * mass exchange Q_ij = G_ij (T_j - T_i) with G_ij = k h dt min(1, min(m_i, m_j) / (rho h^3)),
 * and G2P adds the interpolated node increments Q_i / (m_i cp) to the particles' temperatures.
 * The heat sum m cp T is conserved; dt is limited to 0.9 rho cp h^2 / (6 k). conductivity <= 0
 * turns it off. Applies to scene `scene` (0 for a single-scene handle); not saved in checkpoints. */
int mpm_set_conduction(mpm_handle* h, int32_t scene, double conductivity, double density, double specific_heat);

/* ---- viewer frame (gpu/solver.py:985-1035, the Taichi service's `pack` + `snapshot`) ----
 * One deterministic sample per block of `stride` = ceil(count / preview_limit) caller indices,
 * chosen by the reference's integer hash so previews show no lattice stripes, written as 8 floats
 * per row: x, y, z (m), material index, temperature, pinned, von Mises Kirchhoff stress / J,
 * plastic strain. rows = ceil(count / stride); data holds max_rows x 8 floats. The frame
 * reductions are FP64 on the device. Returns MPM_ERR_NONFINITE, like the reference's snapshot,
 * when any particle's state is not finite. */
typedef struct mpm_frame_info {
  int64_t count, rows, stride;
  double mass, thermal_energy;   /* sum m, sum m cp T */
  double min_T, max_T, min_j, max_von_mises, max_plastic;
  int64_t nonfinite;
  int64_t per_material[256];     /* particles per material index */
} mpm_frame_info;
int mpm_pack_frame(mpm_handle* h, int64_t preview_limit, float* data, int64_t max_rows, mpm_frame_info* info);

/* ---- constitutive batch on the device (projectPlastic + stress, src/three/constitutive.js:52-106)
 * F_in/F_out n x 9, ep/T/dep n, tau n x 9 (Kirchhoff). Stateless; runs on the default stream.
 * Models 2, 3, 8 and 9 carry Jp / dilation between steps and return MPM_ERR_UNSUPPORTED here. */
int mpm_return_map_batch(const mpm_material* material, int64_t n, const double* F_in,
                         const double* ep, const double* T, double dt, double* F_out,
                         double* dep, double* tau);

/* ---- allocation-free particle-to-grid transfer ----
 * No counterpart in the reference. For callers that cannot allocate device memory themselves: a
 * host that owns every device byte through its own pool and passes this library only buffers it
 * already holds, or code running where cudaMalloc is not allowed. Scatters caller-owned device
 * particle arrays onto the domain's grid (stress from F without a return, like the first P2G of an
 * uploaded state: Jp = 1 for snow) and writes, for every node in ((z*ny)+y)*nx+x order, the mass (nx*ny*nz doubles)
 * and the momentum including dt * (stress force + m g) (3*nx*ny*nz doubles): the values
 * mpm_grid_debug returns for the same state. Device pointers: x (n x 3) and F (n x 9 row-major)
 * double; v (n x 3), C (n x 9), m and V float.
 * The intermediate grid lives in one fixed device array of 262,144 nodes (8 MiB) that every GPU
 * which loads the library holds until the process exits; larger grids return MPM_ERR_CAPACITY.
 * The call allocates and frees no device memory. Every call looks up that array's device address
 * on the current device (it stays valid across a device reset); the first call on a device may also
 * load the library's device code, so make it before any stream capture. Every call reuses the same
 * array and clears the nodes it needs first; calls that overlap on the GPU race on it.
 * Launches on `stream` (NULL: the default stream) and returns without waiting. */
int mpm_p2g_noalloc(const mpm_domain* domain, const mpm_material* material, int64_t n, const double* x,
                    const float* v, const double* F, const float* C, const float* m, const float* V,
                    double dt, double* mass, double* momentum, void* stream);

/* ======================================================================================
 * Batched ensembles: many independent scenes stepped by one handle.
 * The reference runs its V&V cases one at a time (src/simulation/vv-mpm.js:30-60 builds and
 * steps one engine per grid phase; src/simulation/vv-benchmarks.js:107-115 solves one sample of
 * an ensemble at a time); these calls replace such loops. Every scene keeps its own domain,
 * grid, material and CFL time step; each substep of the handle advances every scene by its own
 * dt in one launch sequence over all scenes (one persistent G2P2G launch whose work list holds
 * the tiles of every scene). Particles are uploaded and downloaded with mpm_upload_particles /
 * mpm_download_particles as one array in scene order.
 * ====================================================================================== */
typedef struct mpm_scene_desc {
  mpm_domain domain;
  int32_t material;  /* index into the handle's material table (mpm_set_material) */
  int32_t reserved;
  int64_t count;     /* particles of this scene */
} mpm_scene_desc;

typedef struct mpm_tuning {
  int32_t warp_specialised;  /* 1: producer/consumer scatter pass (one 512-thread CTA per SM) */
  int32_t reserved;
  int32_t blocks_per_sm;     /* resident G2P2G CTAs per SM chosen */
  int32_t reorder_interval;  /* substeps between physical re-sorts of the particle state */
  int32_t use_tma;           /* TMA (1) or plain loads (0) for the gather window */
  int32_t trials;            /* configurations timed */
  double ms_per_substep;     /* best configuration */
  double ms_per_substep_default;
} mpm_tuning;

#define MPM_MAX_SCENES 4096
int mpm_batch_create(const mpm_scene_desc* scenes, int32_t nscenes, mpm_handle** out);
int mpm_batch_count(const mpm_handle* h, int32_t* nscenes);
/* nsteps CFL substeps of every scene (each with its own dt). use_graph != 0 replays the
 * substep sequence from a captured CUDA graph (captured on first use, reused while the
 * handle's buffer parity and re-sort phase match). */
int mpm_batch_run(mpm_handle* h, int32_t nsteps, int32_t use_graph);
/* Per-scene simulated time since upload and the dt of the last substep (nscenes each). */
int mpm_batch_times(mpm_handle* h, double* time, double* last_dt);
/* FP64 ledger of one scene (the quantities of mpm_ledger_compute over its particles). */
int mpm_batch_ledger(mpm_handle* h, int32_t scene, mpm_ledger* out);
/* Grid mass and momentum of one scene after P2G (like mpm_grid_debug). */
int mpm_batch_grid_debug(mpm_handle* h, int32_t scene, double dt, double* mass, double* momentum);
/* Autotuner: times trial_substeps substeps for each G2P2G schedule (warp-specialised or not,
 * CTAs per SM, re-sort interval, TMA or plain gather) from the same snapshot of the state, keeps the fastest and
 * restores the state and the scenes' clocks. Works on any handle. */
int mpm_batch_autotune(mpm_handle* h, int32_t trial_substeps, mpm_tuning* out);

/* ======================================================================================
 * Solid position regularisation (src/three/solid-sampling.js:5-42, regularizeSolids): pairs of
 * particles of one material closer than the mean of their target spacings are pushed apart,
 * weighted by inverse mass (pinned particles do not move and have none), with
 *   spacing_i = spacing * cbrt(clamp(V_i det F_i Jp_i / volume_unit, 1/64, 8))
 *   shift     = (x_i - x_j) (target - r) (1 - exp(-rate dt)) / (r (1/m_i + 1/m_j))
 * (coincident pairs along the reference's hashed direction of their indices), every shift of a
 * scene scaled by 1 / max(1, largest |shift| / (max_speed dt)), positions clamped to the domain.
 * Only positions change: v, C, F and the plastic history are kept. The reference's values in its
 * own units are spacing 2.8, volume_unit 1, max_speed 8, rate 40; the reference runs it after
 * every substep unless its solidAntiClump setting is off. Parts are material indices here.
 * ====================================================================================== */
typedef struct mpm_regularizer {
  int32_t enabled;     /* 0: off (the default; mpm_regularize then changes nothing) */
  int32_t reserved;
  double spacing;      /* target spacing (m) of a particle whose V det F Jp equals volume_unit */
  double volume_unit;  /* m^3 */
  double max_speed;    /* displacement budget per second (m/s) */
  double rate;         /* relaxation rate (1/s) */
} mpm_regularizer;
/* Stores the parameters; while enabled, mpm_step / mpm_step_fixed / mpm_step_cfl / mpm_frame_host
 * and batch runs regularise after every substep (as Simulation3.substep does), which splits the
 * fused particle pass into a gather pass, the regularisation and a re-sorted scatter pass. */
int mpm_set_regularizer(mpm_handle* h, const mpm_regularizer* r);
/* One pass now with time step dt (the reference's regularizeSolids(s, dt) after MPM3.step). */
int mpm_regularize(mpm_handle* h, double dt);
/* The same on the caller's positions (x, y, z required; the regularizeSolids(s, dt) drop-in for a
 * host that owns them, like mpm_step_host): copied in, regularised, copied back. */
int mpm_regularize_host(mpm_handle* h, const mpm_particles* io, double dt);

/* ======================================================================================
 * Particle-pair heat exchange and phase change (src/thermal.js:35-56, exchangeHeat, with the
 * pairs of Simulation3.near, src/three/simulation.js:168-174, and the phase change of
 * src/three/phase-change.js:4-18). Every pair of particles of a scene closer than `radius` (and
 * farther than radius * 1.25e-7, the reference's 1e-6 of its 8-unit radius) exchanges
 *   Q = (T_j - T_i) g dt min(b_i, b_j),  g = (1 - r / radius) geometry heat_rate 2 k_i k_j / (k_i + k_j)
 * with b_i = min(1, 0.45 m_i cp_i / (dt sum_j g_ij)) (1 without contacts), applied as +Q / -Q;
 * then h_i += heat_i / m_i, optional ambient loss (T_i - ambient_T) cp_i dt ambient_rate, and the
 * phase decode. A particle that melts or freezes gets the reference's resetParticle (F = I,
 * C = 0, plastic history cleared) and a melted one is unpinned; melted particles keep taking part
 * in the MPM solve here (the reference hands them to its fluid solver; a host does the same with
 * mpm_remove_particle). Reference values in its own units: radius 8 (the neighbour cell),
 * geometry 20, heat_rate 20 (settings.heatRate), ambient_T 15, ambient_rate 0.003.
 * ====================================================================================== */
typedef struct mpm_heat_exchange {
  double radius;        /* m */
  double geometry;      /* m: contact length of the conductance */
  double heat_rate;     /* acceleration factor */
  int32_t ambient;      /* 1: cool toward ambient_T */
  int32_t reserved;
  double ambient_T;
  double ambient_rate;  /* 1/s */
} mpm_heat_exchange;
/* One exchange over the time dt (the reference calls it once per frame with the time advanced).
 * exchanged (may be null): sum over pairs of |Q| (Simulation3.exchangedHeat), FP64. */
int mpm_exchange_heat(mpm_handle* h, const mpm_heat_exchange* x, double dt, double* exchanged);

/* ======================================================================================
 * One domain split into slabs along z (the halo-exchange form of one large scene; no
 * counterpart in the reference, which runs one scene in one worker). Neighbouring slabs hold the
 * same `planes` node planes; after every scatter both copies of a shared node get the sum of both
 * slabs' contributions (only in node tiles the slab has active), so both grid updates give the same
 * velocity there and particles near the seam need no copy. Faces where the domain continues have
 * no wall, no sticky floor and no position clamp. Particles must stay at least 3 node planes inside
 * their slab's grid (no migration here: a host re-partitions by download and upload when needed).
 * ====================================================================================== */
/* On one handle: consecutive scenes of a batch are the slabs (scene s + 1's first `planes` z
 * nodes are scene s's last), every scene takes the same dt (the smallest), and the overlap sum runs
 * after each scatter on the device. */
int mpm_batch_set_slabs(mpm_handle* h, int32_t planes);
/* Across ranks (one single-scene handle per rank): open faces (bit 2 axis + side; z low = 16,
 * z high = 32), a scatter of the current state without stepping, and the overlap planes of the
 * fresh scatter exported to / added from a device buffer of mpm_halo_bytes bytes (16-byte aligned;
 * acc planes then heat planes). A rank exports its side, exchanges buffers with the neighbour,
 * adds what it received, then steps (mpm_step_fixed, one substep, dt = the smallest
 * mpm_stable_dt over ranks). Export and add return after their copy is complete; the caller makes
 * the received buffer ready before mpm_halo_add. */
int mpm_set_open_faces(mpm_handle* h, int32_t faces);
int mpm_prepare(mpm_handle* h);
int mpm_halo_bytes(const mpm_handle* h, int32_t planes, int64_t* bytes);
int mpm_halo_export(mpm_handle* h, int32_t side, int32_t planes, void* device_buffer);
int mpm_halo_add(mpm_handle* h, int32_t side, int32_t planes, const void* device_buffer);

/* ======================================================================================
 * Learned return map. No counterpart in the reference, whose return maps are closed-form or
 * bisection code (src/three/metal-plasticity.js:12-38, src/three/thermal-plasticity.js:12-40):
 * a small MLP (8 -> 64 -> 64 -> 7, ReLU, BF16 tensor-core arithmetic with FP32 accumulation)
 * trained on the GPU from samples of this library's exact J2 / thermal-J2 return, used behind
 * a residual gate that sends every particle it cannot vouch for to the exact map.
 * Inputs (8): the unit direction of the deviatoric trial Hencky strain (Voigt, 6),
 * (T - 293) / 307 and ep / 0.2. Outputs (7): the return in the units of the elastic predictor,
 * (tau - tau_trial) / (2 mu sqrt(3/2) dep_est) (Voigt, 6) and dep / dep_est, with
 * dep_est = (q_trial - sigma_y) J / (3 mu); the projected stress and increment follow exactly
 * from them. Training rows carry a sample weight in column 7 (1 plastic, 0 elastic).
 * Parameters: MPM_SURROGATE_PARAMS floats, W1 [64][16] (inputs 8..15 zero), b1 [64],
 * W2 [64][64], b2 [64], W3 [8][64] (row 7 zero), b3 [8] (entry 7 zero), W[out][in].
 * ====================================================================================== */
#define MPM_SURROGATE_PARAMS 5768
typedef struct mpm_surrogate mpm_surrogate;

typedef struct mpm_surrogate_config {
  int64_t samples;       /* training set drawn once from the exact map */
  int32_t batch;         /* minibatch, a multiple of 16 */
  int32_t steps;         /* AdamW steps */
  double lr, weight_decay;
  double dep_weight;     /* loss weight of the dep output (others 1) */
  int32_t cosine;        /* 1: cosine learning-rate decay */
  int32_t newton;        /* Johnson-Cook: most Newton steps after the prediction (0: 8) */
  uint64_t seed;
  double strain_min, strain_max; /* log-uniform magnitude of the principal trial log strains */
  double T_min, T_max, ep_max;   /* uniform temperature and plastic strain */
  double dt_min, dt_max;         /* Johnson-Cook: log-uniform substep (0, 0: 1e-7 .. 1e-5 s) */
} mpm_surrogate_config;

typedef struct mpm_gate_counts {
  uint32_t elastic;   /* below yield: exact elastic branch */
  uint32_t learned;   /* prediction accepted by the gate */
  uint32_t fallback;  /* prediction rejected: exact return */
  uint32_t reserved;
} mpm_gate_counts;

int mpm_surrogate_create(const mpm_material* material, uint64_t seed, mpm_surrogate** out);
int mpm_surrogate_destroy(mpm_surrogate* s);
const char* mpm_surrogate_last_error(const mpm_surrogate* s);
int mpm_surrogate_get_weights(mpm_surrogate* s, float* params);
int mpm_surrogate_set_weights(mpm_surrogate* s, const float* params);
/* n training rows from the exact map (X n x 8 features, Y n x 8 targets, column 7 zero); with F
 * non-null also the trial states (F n x 9, ep, T). */
int mpm_surrogate_samples(mpm_surrogate* s, const mpm_surrogate_config* cfg, int64_t n, float* X, float* Y, double* F,
                          double* ep, double* T);
/* Draws cfg->samples rows and runs cfg->steps AdamW steps on the GPU; loss_history (steps
 * floats, may be NULL) receives the weighted mean squared error of each minibatch. */
int mpm_surrogate_train(mpm_surrogate* s, const mpm_surrogate_config* cfg, float* loss_history);
/* Gradient of the weighted mean squared error over n rows (n a multiple of 16) at the current
 * weights, from the same forward/backward kernel training uses (no update). */
int mpm_surrogate_grad(mpm_surrogate* s, int64_t n, const float* X, const float* Y, const float* out_weight,
                       float* grad, double* loss);
int mpm_surrogate_forward(mpm_surrogate* s, int64_t n, const float* X, float* Y);
/* Return map of n trial states (F n x 9 row-major, ep, T) through the gate: F_out n x 9,
 * dep n, tau n x 9 (Kirchhoff), path n (0 elastic, 1 learned, 2 exact fallback; may be NULL).
 * use_mlp = 0 runs the exact map for every particle through the same kernel. */
int mpm_return_map_learned(mpm_surrogate* s, int64_t n, const double* F_in, const double* ep, const double* T,
                           double gate_tol, int32_t use_mlp, double* F_out, double* dep, double* tau, int8_t* path,
                           mpm_gate_counts* counts);
/* ---- learned return map inside the step ----
 * The reference's per-particle return (src/three/mpm.js:126-131 calling projectPlastic,
 * src/three/constitutive.js:52-78) with the Johnson-Cook plastic increment
 * (src/three/metal-plasticity.js:28-34, 24 bisection halvings of the consistency condition) taken from a
 * network trained for models 6 / 7 (mpm_surrogate_create with such a material, mpm_surrogate_train):
 * the fused particle pass evaluates it on the tensor cores for every particle whose trial stress
 * exceeds the initial flow stress, refines the predicted increment by at most `newton` Newton steps
 * on the consistency condition (stopping once the gate passes) and accepts it only when the
 * dimensionless residual |q - 3 mu / J dep - flow(ep + dep, dep / dt, T)| / q is at most gate_tol
 * (the stress residual is then at most gate_tol x the trial stress); every other particle takes the
 * exact bisection. The handle keeps its own copy of the weights (the surrogate may be destroyed
 * afterwards). MPM_RETURN_EXACT restores the reference's map. Scenes with grid conduction or with
 * snow, sand or pressure materials run the exact map (MPM_ERR_UNSUPPORTED when set on such a
 * handle). Batch handles take it for all their scenes. */
#define MPM_RETURN_EXACT 0
#define MPM_RETURN_LEARNED_GATED 1
/* The same refinement and gate without a network (s may be NULL): the Newton steps start from the
 * root of the rate- and hardening-free condition, u0 = 1 - flow(ep, 0, T) / q. */
#define MPM_RETURN_NEWTON_GATED 2
int mpm_set_return_mode(mpm_handle* h, int32_t mode, mpm_surrogate* s, double gate_tol, int32_t newton);
/* Returns served by the network (learned) and sent to the exact map (fallback) since the mode was
 * set or the counts were last reset (reset != 0 clears them after the read); elastic is 0. */
int mpm_gate_counts_read(mpm_handle* h, mpm_gate_counts* out, int32_t reset);

/* Device time per call of the gated map and of the exact map on n device-resident random trial
 * states drawn like cfg's training set (iters calls each, CUDA events). */
int mpm_surrogate_time(mpm_surrogate* s, const mpm_surrogate_config* cfg, int64_t n, int32_t iters, double gate_tol,
                       double* ms_exact, double* ms_learned, mpm_gate_counts* counts);
/* The same random Johnson-Cook states through the Newton-gated map without the network (the
 * refinement and gate of the learned map from u0 = 1 - flow(ep, 0, T) / q, the bisection for what the
 * gate rejects): device time per call; counts as above (learned = accepted). */
int mpm_surrogate_time_newton(mpm_surrogate* s, const mpm_surrogate_config* cfg, int64_t n, int32_t iters,
                              double gate_tol, double* ms, mpm_gate_counts* counts);

/* ======================================================================================
 * 2D elastic solid: drop-in for the reference's SolidMPM (src/solid-mpm.js:20-116).
 * Fixed 149 x 149 node grid, DX = 8, origin -592 (src/solid-mpm.js:4); fixed-corotated
 * elasticity with E = rho * 16000 * solidStiffness and mu = lambda = 0.4 E. The handle owns
 * F and C on the device (the reference's f00..c11 fields); the caller owns the particle
 * arrays and passes them with every call, like `s` in the reference (host pointers, copied
 * in and, for x/y/vx/vy, back out).
 * ====================================================================================== */
#define SMPM_SCENE_OTHER 0
#define SMPM_SCENE_SOFTBODY 1 /* s.scene === 'softbody' (src/solid-mpm.js:65) */
#define SMPM_SCENE_BASIN 2    /* s.scene === 'basin' */
#define SMPM_GRAVITY_NONE 0
#define SMPM_GRAVITY_CENTER 1 /* settings.gravity 'center' (src/simulation.js:276-278) */
#define SMPM_GRAVITY_UNIFORM 2

/* The caller's particle arrays and the settings the step reads (src/simulation.js:18-31). */
typedef struct smpm_sim {
  int32_t count;
  int32_t scene;             /* SMPM_SCENE_* */
  int32_t boundary;          /* settings.boundary */
  int32_t gravity;           /* SMPM_GRAVITY_*; read by smpm_frame only */
  double solid_stiffness;    /* settings.solidStiffness */
  double strength;           /* settings.strength; read by smpm_frame only */
  float *x, *y, *vx, *vy;    /* in/out */
  const float *mass, *volume;
  const uint8_t *material, *pinned;
} smpm_sim;

typedef struct smpm_stats { /* SolidMPM.stats (src/solid-mpm.js:108-116) */
  int32_t count;
  int32_t nodes;
  int32_t substeps;
  int32_t pad;
  double min_j, max_j, strain;
} smpm_stats;

typedef struct smpm_handle smpm_handle;

/* new SolidMPM(capacity) (src/solid-mpm.js:21-25): F = I, C = 0 for every slot. */
int smpm_create(int64_t capacity, smpm_handle** out);
int smpm_destroy(smpm_handle* h);
const char* smpm_last_error(const smpm_handle* h);
/* Material ids treated as MPM solids (MATERIALS[m].mpm, src/solid-mpm.js:7); default {11}. */
int smpm_set_mpm_materials(smpm_handle* h, const uint8_t* ids, int32_t n);
int smpm_reset(smpm_handle* h);                                   /* SolidMPM.reset */
int smpm_reset_particle(smpm_handle* h, int64_t i);               /* SolidMPM.resetParticle */
int smpm_remove_particle(smpm_handle* h, int64_t i, int64_t last); /* SolidMPM.removeParticle */
int smpm_has_particles(smpm_handle* h, const smpm_sim* s, int32_t* out); /* SolidMPM.hasParticles */
int smpm_stable_step(smpm_handle* h, const smpm_sim* s, double* dt);     /* SolidMPM.stableStep */
int smpm_step(smpm_handle* h, const smpm_sim* s, double dt);             /* SolidMPM.step */
int smpm_stats_get(smpm_handle* h, const smpm_sim* s, smpm_stats* out);  /* SolidMPM.stats */
/* The MPM branch of Simulation.step (src/simulation.js:246-254) for a simulation whose moving
 * particles are all MPM solids, on the device: up to 96 substeps of h = min(remaining,
 * stableStep), each applying the body force of Simulation.substep (src/simulation.js:270-288)
 * before the step. dt is clamped to [0, 0.05]. One host round trip per call. */
int smpm_frame(smpm_handle* h, const smpm_sim* s, double dt, int32_t* substeps, double* advanced);
/* Read / write the eight deformation fields (f00 f01 f10 f11 c00 c01 c10 c11) of slots
 * [0, n) as fields[8][n] doubles. */
int smpm_get_fields(smpm_handle* h, int64_t n, double* fields);
int smpm_set_fields(smpm_handle* h, int64_t n, const double* fields);

#ifdef __cplusplus
}
#endif
#endif /* MPM_B200_H */
