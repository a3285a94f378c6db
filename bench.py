#!/usr/bin/env python
"""Benchmark of the B200-native MLS-MPM solid step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workload (default): the 2,097,152-particle J2 linear-hardening drop (64x64x64-cell block, 8 particles
per cell, 128^3 grid, aluminium E=70 GPa, nu=0.33, yield 250 MPa, hardening 1 GPa), seeded
synthetic input. One step = one requested step of dt=2e-6 s, sub-stepped on the device to CFL 0.4
(about 4 substeps); the metric counts actual substeps x particles. The K timed steps go through
mpm_run (one call, the step boundaries taken on the device); "step_per_call" gives the same steps as
K mpm_step calls. Multi-GPU runs are independent replicas per GPU (weak scaling), or with --slabs
one scene split into z slabs (strong scaling).

The line also carries an "ensemble" block: 256 seeded V&V scenes (particle counts log-uniform in
5e3..2e5, grids 32..96 cells, per-scene CFL dt) on one batch handle per rank, scenes sharded across
ranks by cost, against the plain form with one handle per scene (--no-ensemble skips it,
--ensemble-only runs only it), and at N=1 a "surrogate" block: the learned return map trained on
the GPU and timed, gated, against the exact map (--no-surrogate skips it).

--impl reference times the reference's CPU algorithm (the FP64 port under oracle/, all host threads,
because the reference itself is JavaScript and no JS runtime exists here) on a bounded sub-block
of the same workload and prints the same JSON line with "impl": "reference".
"""
import argparse
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "summer-particle-lab_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "particle-steps/s, 2M-particle J2 MPM: surrogate+batched vs exact, same stress err"
UNIT = "particle-steps/s"
# algorithmic bytes per particle-step (FP32 state read once and written once) and per active node
BYTES_PER_PARTICLE = {0: 200, 1: 200, 4: 208, 5: 208, 6: 216, 7: 208, 10: 216}
BYTES_PER_NODE = 56


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="j2_drop")
    ap.add_argument("--shape", default="64,64,64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--clocks-csv", default=None, help="also write the clock samples to this CSV file")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--surrogate-only", action="store_true")
    ap.add_argument("--learned-newton", type=int, default=8, help="most Newton steps after the network's prediction")
    ap.add_argument("--learned-gate", type=float, default=1e-5, help="gate: consistency residual / trial stress")
    ap.add_argument("--surrogate-steps", type=int, default=0, help="training steps (0: the default schedule)")
    ap.add_argument("--ensemble-only", action="store_true")
    ap.add_argument("--ensemble-scenes", type=int, default=256)
    ap.add_argument("--ensemble-steps", type=int, default=64)
    ap.add_argument("--no-autotune", action="store_true",
                    help="ensemble: keep the default schedule (2 CTAs/SM, TMA, re-sort every 32 substeps) "
                         "instead of timing the candidates first (for profiling a known launch sequence)")
    ap.add_argument("--slabs", action="store_true",
                    help="N > 1: split the one scene into N slabs along z with an overlap exchange per substep "
                         "(strong scaling) instead of N replicas")
    return ap.parse_args()


def make_scene(args):
    from mpm_b200 import scenes
    if args.workload == "j2_drop":
        shape = tuple(int(s) for s in args.shape.split(","))
        return scenes.j2_drop(shape=shape)
    if args.workload == "j2_drop_plastic":
        shape = tuple(int(s) for s in args.shape.split(","))
        return scenes.j2_drop(shape=shape, plastic=True)
    if args.workload == "elastic_cube":
        return scenes.elastic_cube()
    if args.workload == "thermal_j2":
        return scenes.thermal_j2()
    if args.workload == "coupled_collision":
        return scenes.coupled_collision()
    if args.workload == "jc_impact":
        return scenes.jc_impact()
    raise SystemExit(f"unknown workload {args.workload}")


def sample_scene(scene, factor=2):
    """A sub-block of the scene (every axis of the block divided by factor), same grid/material."""
    from mpm_b200 import scenes
    x = scene.x
    d = scene.domain
    lo = x.min(0)
    hi = x.max(0)
    ext = (hi - lo) / factor
    keep = np.all(x <= lo + ext + 1e-12, axis=1)
    s = scenes.Scene(name=scene.name + "_sample", domain=d, materials=scene.materials, x=x[keep].copy(),
                     v=scene.v[keep].copy(), m=scene.m[keep].copy(), V=scene.V[keep].copy(),
                     mat=scene.mat[keep].copy(), T=None if scene.T is None else scene.T[keep].copy(),
                     meta=dict(scene.meta))
    return s


def oracle_requested_step(st, dt_req, threads, max_substeps=48):
    """One requested step on the oracle, sub-stepped as Simulation3.step does
    (src/three/simulation.js:305-311): substeps of the stable dt, the last one taking what is left."""
    left, n = dt_req, 0
    while left > 1e-6 * dt_req and n < max_substeps:
        dt = min(st.stable_dt(), left)
        if left - dt <= 1e-6 * dt_req:
            dt = left
        st.step(dt, threads=threads)
        left -= dt
        n += 1
    return n


def cpu_oracle_rate(scene, dt_req, steps, threads, budget_s=None):
    """Oracle particle-steps/s on the given scene: `steps` requested steps of dt_req sub-stepped to
    the stable dt (OpenMP threads), stopping early once budget_s seconds have passed. Returns
    (rate, seconds, requested steps timed, substeps)."""
    from oracle import oracle as orc
    st = orc.state_from_scene(scene)
    oracle_requested_step(st, dt_req, threads)  # warm-up
    t0 = time.perf_counter()
    done = subs = 0
    while done < steps:
        subs += oracle_requested_step(st, dt_req, threads)
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    return scene.n * subs / el, el, done, subs


class Clocks:
    """SM clocks, power and clock-event reasons sampled during the run: an NVML thread every 20 ms
    (read-only queries), or `nvidia-smi -lms 100` when NVML is unavailable. Samples stay in memory;
    with --clocks-csv PATH they are also written there with their host time (nvidia-smi writes its
    rows to that path, or to a temporary file)."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index, path=None):
        self.index = index
        self.proc = None
        self.thread = None
        self.rows = []  # (time, sm_mhz, max_mhz, power_w, [active reason names])
        self.keep = path is not None
        if path is None:
            import tempfile
            fd, path = tempfile.mkstemp(prefix="clocks_bench_", suffix=".csv")
            os.close(fd)
        self.path = path

    def wait_first_sample(self, timeout=5.0):
        t0 = time.time()
        while time.time() - t0 < timeout:
            if self.rows or (self.proc is not None and os.path.exists(self.path) and os.path.getsize(self.path) > 0):
                return
            if self.thread is None and self.proc is None:
                return
            time.sleep(0.02)

    def _nvml_loop(self, nv, h):
        bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        while not self.stop:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1e3
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((time.time(), float(sm), float(mx), pw, [n for n, b in zip(self.NAMES, bits) if rs & b]))
            except Exception:
                pass
            time.sleep(0.02)

    def __enter__(self):
        if os.path.dirname(self.path):
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.stop = False
            self.thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            self.t0 = time.time()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self.stop = True
            self.thread.join(timeout=2)
            if self.keep:
                with open(self.path, "w") as f:
                    f.write("time,sm_mhz,max_sm_mhz,power_w,reasons\n")
                    for t, sm, mx, pw, rs in self.rows:
                        f.write(f"{t:.3f},{sm:.0f},{mx:.0f},{pw:.1f},{'|'.join(rs) or 'none'}\n")
            elif os.path.exists(self.path):
                os.remove(self.path)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, t_start=None, t_end=None):
        """Median SM clock, max clock and the reasons seen in the samples taken during [t_start,
        t_end] (the timed region)."""
        if self.thread is not None:
            rows = [r for r in self.rows if t_start is None or t_start <= r[0] <= t_end]
            if not rows:  # a region shorter than the sampling period: the samples on either side
                before = [r for r in self.rows if r[0] < t_start][-1:]
                after = [r for r in self.rows if r[0] > t_end][:1]
                rows = before + after
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
            sm = sorted(r[1] for r in rows)
            return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[2] for r in rows),
                    "reasons": sorted({n for r in rows for n in r[4]}), "samples": len(rows),
                    "power_w_median": sorted(r[3] for r in rows)[len(rows) // 2], "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows_all = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows_all.append(parts)
        # nvidia-smi -lms prints one row per period from t0; map row i to t0 + (i + 1) * period
        rows = rows_all
        if t_start is not None and rows_all:
            per = 0.1
            sel = [r for i, r in enumerate(rows_all) if t_start - per <= self.t0 + (i + 1) * per <= t_end + per]
            rows = sel if sel else rows_all[-2:]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        reasons = sorted({self.NAMES[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi"}


# DRAM bytes per particle of one fused G2P2G launch (dram__bytes_read.sum + dram__bytes_write.sum of
# one ncu --set full capture of k_particles<1,0,0> on the 2M-particle J2 drop, divided by the particle
# count), set by hand from that capture; bench.py scales it to the timed workload's particle count.
TRAFFIC_PER_PARTICLE = 153.9
TRAFFIC_SOURCE = "ncu --set full capture of k_particles<1,0,0,0>, j2_drop 2,097,152 particles (322.8 MB per launch)"


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def run_reference(args, rank, world):
    """The reference's CPU algorithm (the FP64 port of src/three/mpm.js under oracle/, built with
    -march=native on this host, all host threads) on a 1/8 sub-block of the same workload, each step
    a requested step of the workload's dt sub-stepped to the stable dt like Simulation3.step; the
    metric counts particles x substeps like the GPU arm. Bounded to about 90 s of timed work."""
    if rank != 0:
        return
    from oracle import oracle as orc
    isa = orc.use_native()
    scene = make_scene(args)
    sample = sample_scene(scene, 2)
    threads = os.cpu_count() or 1
    dt_req = scene.meta.get("dt", 2e-6)
    st = orc.state_from_scene(sample)
    for _ in range(max(1, args.warmup)):
        oracle_requested_step(st, dt_req, threads)
    t0 = time.perf_counter()
    done = subs = 0
    while done < args.steps:
        subs += oracle_requested_step(st, dt_req, threads)
        done += 1
        if time.perf_counter() - t0 > 90.0:
            break
    el = time.perf_counter() - t0
    value = sample.n * subs / el
    sample_desc = (f"{sample.n}-particle sub-block (1/8) of {scene.meta['workload']}, {done} requested steps of "
                   f"{dt_req} s ({subs} CFL substeps) in {el:.1f} s")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / max(done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": scene.meta["workload"], "sample_particles": sample.n,
                       "dt_requested": dt_req, "steps_timed": done, "substeps_timed": subs},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "isa": isa,
                             "sample": sample_desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def ensemble_leg(args, rank, world, dist):
    """The V&V ensemble (seeded scenes with log-uniform particle counts 5e3..2e5, grids 32..96 cells,
    E, nu, yield drawn per scene, CFL 0.4 dt per scene): scenes sharded across ranks by cost; each
    rank steps its scenes on one batch handle (autotuned schedule, substeps replayed from a CUDA
    graph), timed with CUDA events on the library stream. The plain form steps the same scenes
    with one single-scene handle each, round-robin, one CFL substep per call (wall clock around
    the loop, synchronized). Both count particles x substeps."""
    import torch
    from mpm_b200 import scenes
    from mpm_b200.ensemble import gather_ledgers, imbalance, ledger_rows, scene_cost, shard_scenes
    from mpm_b200.solver import Batch, Solver
    allsc = scenes.ensemble(args.ensemble_scenes)
    costs = [scene_cost(sc) for sc in allsc]
    shards = shard_scenes(costs, world)
    idx = shards[rank]
    mine = [allsc[k] for k in idx]
    K = args.ensemble_steps

    def max_sum(ms, parts):
        t = torch.tensor([ms, parts], dtype=torch.float64, device="cuda")
        if dist is not None:
            dist.all_reduce(t[0:1], op=dist.ReduceOp.MAX)
            dist.all_reduce(t[1:2], op=dist.ReduceOp.SUM)
        return float(t[0]), float(t[1])

    n_mine = sum(sc.n for sc in mine)
    b = Batch(mine)
    b.upload()
    tune = b.autotune(6) if not args.no_autotune else {"skipped": "default schedule (--no-autotune)"}
    b.run(K, graph=True)  # warm-up, captures the graph
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ext = torch.cuda.ExternalStream(b.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = b.launch_count()
    e0.record(ext)
    b.run(K, graph=True)
    e1.record(ext)
    torch.cuda.synchronize()
    launches = b.launch_count() - l0
    ms, psteps = max_sum(e0.elapsed_time(e1), n_mine * K)
    batched = {"value": psteps / (ms / 1e3), "ms_per_substep": ms / K, "substeps": K, "cuda_graph": True,
               "gpu_launches": launches, "tuning": tune}
    # roofline of the batched G2P2G from an eagerly profiled stretch
    b.profile(True)
    b.run(8, graph=False)
    prof = b.profile_read()
    b.profile(False)
    g_ms, g_n = prof["g2p2g"]
    active = 0
    for k, sc in enumerate(mine):
        gm, _ = b.scene_grid_debug(k, 1e-7)
        active += int(np.count_nonzero(gm > 0))
    alg = sum(sc.n * BYTES_PER_PARTICLE[sc.materials[0].model] for sc in mine) + BYTES_PER_NODE * active
    hbm, peak_kind = peaks()
    ach = alg / (g_ms / g_n / 1e3) / 1e9 if g_n else None
    ledgers = gather_ledgers(ledger_rows(b, idx), idx, len(allsc), dist)
    b.close()
    # plain: one handle per scene
    handles = []
    for sc in mine:
        h = Solver(sc.domain, sc.n)
        h.upload(sc)
        h.step_cfl(1)
        handles.append(h)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    Kp = max(2, K // 8)
    t0 = time.perf_counter()
    for _ in range(Kp):
        for h in handles:
            h.step_cfl(1)
    torch.cuda.synchronize()
    pms, pp = max_sum((time.perf_counter() - t0) * 1e3, n_mine * Kp)
    # the same substeps again with CUDA events around every launch on each handle's stream: the sum
    # of the kernel durations is the device time the plain form needs without its host loop
    for h in handles:
        h.profile(True)
    for _ in range(Kp):
        for h in handles:
            h.step_cfl(1)
    torch.cuda.synchronize()
    dev_ms = 0.0
    for h in handles:
        dev_ms += sum(v[0] for v in h.profile_read().values())
        h.profile(False)
    dms, _ = max_sum(dev_ms, 0.0)
    for h in handles:
        h.close()
    plain = {"value": pp / (pms / 1e3), "ms_per_substep": pms / Kp, "substeps": Kp, "handles": len(allsc),
             "timing": "wall clock around the host loop",
             "device_value": pp / (dms / 1e3), "device_ms_per_substep": dms / Kp,
             "device_timing": "sum of CUDA-event kernel durations on every handle's stream (no host loop)"}
    return {"workload": f"vv_ensemble_{len(allsc)}_seeds_1000", "scenes": len(allsc),
            "particles": int(sum(sc.n for sc in allsc)), "ranks": world,
            "shard_imbalance": imbalance(costs, shards), "batched": batched, "plain": plain,
            "speedup_batched_vs_plain": batched["value"] / plain["value"],
            "speedup_batched_vs_plain_device": batched["value"] / plain["device_value"],
            "roofline": {"bound": "hbm", "kernel": "k_g2p2g (all scenes)", "achieved": ach, "peak": hbm,
                         "unit": "GB/s", "frac": ach / hbm if ach else None,
                         "algorithmic_bytes_per_launch": alg, "launch_ms": g_ms / g_n if g_n else None,
                         "peak_source": peak_kind},
            "ledger_total_mass": float(ledgers[:, 0].sum()), "ledger_min_j": float(ledgers[:, 5].min())}


def surrogate_leg(steps=0):
    """Learned return map on the thermo-elastoplastic law (J2, yield 250 MPa softening 0.3 MPa/K):
    training on the GPU (10M exact-map samples, BF16 tensor-core forward/backward, AdamW), then
    the gated map against the exact map on 4,096,000 device-resident trial states (trial log
    strains log-uniform 1e-5..5e-2, random directions, T 293..600 K, ep 0..0.2), CUDA events."""
    import torch
    from mpm_b200 import scenes
    from mpm_b200.params import MODEL_THERMAL_J2
    from mpm_b200.surrogate import Surrogate, config
    T_ref, hot = 293.0, 0.001
    mat = scenes.aluminium_j2(MODEL_THERMAL_J2, T_ref=T_ref, T_hot=T_ref + (1 - hot) * 250e6 / 0.3e6, hot_ratio=hot,
                              heat_fraction=0.9, specific_heat=900.0)
    s = Surrogate(mat, seed=5)
    cfg = config(steps=steps) if steps > 0 else config()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = s.train(cfg)
    el = time.perf_counter() - t0
    mlp_flop = 2 * (8 * 64 + 64 * 64 + 64 * 7)  # forward per sample; backward is about twice that
    train_flops = 3.0 * mlp_flop * cfg.batch * cfg.steps
    bf16_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"] if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else 1590.0
    n = 4_096_000
    rows = []
    for tol in (2e-3, 5e-3, 1e-2):
        r = s.time(n, iters=10, gate_tol=tol)
        plastic = r["learned"] + r["fallback"]
        rows.append({"gate_tol": tol, "stated_stress_error_of_accepted": f"{4 * tol:g} x yield",
                     "ms_exact": r["ms_exact"], "ms_gated": r["ms_learned"],
                     "speedup_gated_vs_exact": r["ms_exact"] / r["ms_learned"],
                     "elastic": r["elastic"], "learned": r["learned"], "fallback": r["fallback"],
                     "learned_share_of_plastic": r["learned"] / plastic if plastic else None})
    s.close()
    return {"law": "thermal J2 (model 10), E 70 GPa, nu 0.33, yield 250 MPa, H 1 GPa, -0.3 MPa/K",
            "network": "8-64-64-7 ReLU, BF16 operands, FP32 accumulate; training and the gated map on tcgen05 "
                       "(TMEM accumulators, 128 samples per tile)",
            "training": {"samples": cfg.samples, "batch": cfg.batch, "steps": cfg.steps, "seconds": el,
                         "loss_first": float(hist[:10].mean()), "loss_last": float(hist[-100:].mean()),
                         "mlp_tflops": train_flops / el / 1e12,
                         "tensor_frac_of_measured_bf16": train_flops / el / 1e12 / bf16_peak,
                         "note": "wall clock of the whole call, sample generation included"},
            "return_map_4096000_states": rows,
            "exact_stress_error": "FP32 exact map: within 1e-5 x yield of the FP64 oracle (tests/test_surrogate.py)"}


def learned_step_leg(args):
    """The learned return map inside the fused step, on the law whose exact return iterates: a
    Johnson-Cook network (8-64-64-7, BF16 tensor cores, FP32 accumulation) trained on the GPU from
    the exact bisection's roots, then
      - the 2M-particle Johnson-Cook impact (64^3-cell block, 8 ppc, 128^3 grid, 60 m/s) stepped K
        requested steps through mpm_run in exact and in learned mode from the same initial state
        (CUDA events on the handle's stream), and
      - the 256-scene V&V ensemble with Johnson-Cook materials on one batch handle with graph replay,
        exact and learned,
    both at one stated stress error: the gate accepts a prediction only when its consistency
    residual is at most gate_tol x the trial stress (the bisection's own FP32 residual is below it);
    the end states of the modes are compared. Beside them the same refinement and gate without the
    network (newton_gated: Newton from the initial flow stress's guess), what the network is
    measured against."""
    import torch
    from mpm_b200 import scenes
    from mpm_b200.solver import Batch, Solver
    from mpm_b200.surrogate import Surrogate, jc_config
    gate_tol, newton = args.learned_gate, args.learned_newton
    mat = scenes.johnson_cook_metal(7)
    s = Surrogate(mat, seed=11)
    cfg = jc_config(newton=newton)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = s.train(cfg)
    train_s = time.perf_counter() - t0
    kern = s.time(4_096_000, iters=10, gate_tol=gate_tol, cfg=cfg)
    kern_nw = s.time_newton(4_096_000, iters=10, gate_tol=gate_tol, cfg=cfg)
    plastic_k = kern["learned"] + kern["fallback"]
    scene = scenes.jc_impact()
    dt_req = scene.meta["dt"]
    K = args.steps

    def timed(mode):
        sol = Solver(scene.domain, scene.n)
        sol.upload(scene)
        if mode == "learned":
            sol.set_return_mode(s, gate_tol=gate_tol, newton=newton)
        elif mode == "newton":
            sol.set_return_mode(mode="newton", gate_tol=gate_tol, newton=newton)
        ext = torch.cuda.ExternalStream(sol.stream())
        sol.run(dt_req, max(1, args.warmup))
        sol.gate_counts(reset=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        sub, _ = sol.run(dt_req, K)
        e1.record(ext)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        counts = sol.gate_counts()
        out = sol.download(("x", "ep", "F"))
        st = sol.status()
        sol.close()
        return {"value": scene.n * sub / (ms / 1e3), "ms_per_step": ms / K, "substeps": sub, "status": st,
                "gate_learned": counts[0], "gate_fallback": counts[1]}, out

    ex, ox = timed(None)
    le, ol = timed("learned")
    ne, on = timed("newton")
    served = le["gate_learned"] / max(1, le["gate_learned"] + le["gate_fallback"])
    step = {"workload": scene.meta["workload"], "particles": scene.n, "requested_steps": K, "dt_requested": dt_req,
            "exact": ex, "learned": le, "speedup_learned_vs_exact": le["value"] / ex["value"],
            "learned_share_of_returns": served,
            "newton_gated": ne, "speedup_newton_vs_exact": ne["value"] / ex["value"],
            "newton_share_of_returns": ne["gate_learned"] / max(1, ne["gate_learned"] + ne["gate_fallback"]),
            "newton_end_state_difference": {"x_m": float(np.max(np.abs(ox["x"] - on["x"]))),
                                            "ep": float(np.max(np.abs(ox["ep"] - on["ep"])))},
            "end_state_difference": {"x_m": float(np.max(np.abs(ox["x"] - ol["x"]))),
                                     "ep": float(np.max(np.abs(ox["ep"] - ol["ep"]))),
                                     "F": float(np.max(np.abs(ox["F"] - ol["F"]))),
                                     "max_ep": float(np.max(ox["ep"]))}}
    # the V&V ensemble with Johnson-Cook materials on one batch handle, exact and learned
    ens = scenes.ensemble(args.ensemble_scenes, model=7)
    Ke = args.ensemble_steps
    n_all = sum(sc.n for sc in ens)

    def batch_run(mode):
        b = Batch(ens)
        b.upload()
        if mode == "learned":
            b.set_return_mode(s, gate_tol=gate_tol, newton=newton)
        elif mode == "newton":
            b.set_return_mode(mode="newton", gate_tol=gate_tol, newton=newton)
        b.run(Ke, graph=True)  # warm-up, captures the graph
        b.gate_counts(reset=True)
        torch.cuda.synchronize()
        ext = torch.cuda.ExternalStream(b.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        b.run(Ke, graph=True)
        e1.record(ext)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        counts = b.gate_counts()
        st = b.status()
        b.close()
        return {"value": n_all * Ke / (ms / 1e3), "ms_per_substep": ms / Ke, "status": st,
                "gate_learned": counts[0], "gate_fallback": counts[1]}

    bex = batch_run(None)
    ble = batch_run("learned")
    bne = batch_run("newton")
    s.close()
    mlp_flop = 2 * (8 * 64 + 64 * 64 + 64 * 7)
    return {"law": "Johnson-Cook model 7 (A = B = yield, n 0.35, C 0.025, rate0 1/s; src/three/metal-plasticity.js:28-34, "
                   "24 bisection halvings)",
            "network": "8-64-64-7 ReLU: training on tcgen05 (TMEM accumulators); in-step inference as warp-wide "
                       "mma.sync m16n8k16 tiles inside the fused pass, FP32 accumulate",
            "gate": {"tol": gate_tol, "newton_steps_max": newton,
                     "stated_stress_error": f"consistency residual <= {gate_tol:g} x trial stress for every accepted "
                                            f"return"},
            "training": {"samples": cfg.samples, "batch": cfg.batch, "steps": cfg.steps, "seconds": train_s,
                         "loss_first": float(hist[:10].mean()), "loss_last": float(hist[-100:].mean()),
                         "mlp_tflops": 3.0 * mlp_flop * cfg.batch * cfg.steps / train_s / 1e12,
                         "note": "wall clock of the whole call, sample generation included"},
            "return_map_4096000_states": {"ms_exact": kern["ms_exact"], "ms_learned": kern["ms_learned"],
                                          "speedup": kern["ms_exact"] / kern["ms_learned"],
                                          "learned_share_of_plastic": kern["learned"] / max(1, plastic_k),
                                          "plastic": plastic_k,
                                          "ms_newton_gated": kern_nw["ms"],
                                          "speedup_newton_vs_exact": kern["ms_exact"] / kern_nw["ms"],
                                          "newton_share_of_plastic": kern_nw["accepted"] / max(
                                              1, kern_nw["accepted"] + kern_nw["fallback"])},
            "step": step,
            "ensemble": {"workload": f"vv_ensemble_jc_{len(ens)}_seeds_1000", "particles": n_all, "substeps": Ke,
                         "exact_batched": bex, "learned_batched": ble, "newton_gated_batched": bne,
                         "speedup_learned_vs_exact": ble["value"] / bex["value"],
                         "speedup_newton_vs_exact": bne["value"] / bex["value"]}}


def slab_leg(args, rank, world, dist):
    """The single scene split into `world` slabs along z, one per GPU, its overlap planes exchanged
    with NCCL after every substep (host-driven substeps at the smallest CFL dt over ranks)."""
    import torch
    from mpm_b200.slabs import SlabRank, partition, slab_domains
    scene = make_scene(args)
    planes = 6
    slabs = slab_domains(scene.domain, world, planes)
    part, _ = partition(scene, slabs)[rank]

    class Buf:
        def __init__(self, nbytes):
            self.t = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
            self.ptr = self.t.data_ptr()

    def transport(send, recv, peer):
        ops = [dist.P2POp(dist.isend, send.t, peer), dist.P2POp(dist.irecv, recv.t, peer)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        torch.cuda.synchronize()

    def reduce_min(x):
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        return float(t.item())

    sr = SlabRank(part, slabs[rank], rank, world, planes, transport, reduce_min, Buf)
    ext = torch.cuda.ExternalStream(sr.solver.stream())
    dt_req = scene.meta.get("dt", 2e-6)
    for _ in range(args.warmup):
        sr.advance(dt_req)
    torch.cuda.synchronize()
    dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    substeps = sum(sr.advance(dt_req) for _ in range(args.steps))
    e1.record(ext)
    torch.cuda.synchronize()
    dist.barrier()
    t = torch.tensor([e0.elapsed_time(e1) / 1e3], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    elapsed = float(t.item())
    status = sr.solver.status()
    sr.close()
    if rank != 0:
        return
    value = scene.n * substeps / elapsed
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": scene.meta.get("workload"), "particles": scene.n, "parallelism": f"slabs{world} along z",
                   "shared_planes": planes, "dt_requested": dt_req, "substeps_per_step": substeps / args.steps,
                   "timing": "CUDA events on the slab handle's stream around the host-driven substep loop "
                             "(one NCCL exchange and one dt all-reduce per substep), max over ranks"},
        "status": status}), flush=True)


def e2e_leg(args, sol, scene, dt_req, ext, dist, dtype):
    """K requested steps through mpm_frame_host with the caller's positions and velocities in pinned
    host arrays of `dtype`: every step copies them to the device, steps, and copies them back inside
    the timed region (CUDA events on the handle's stream, max over ranks)."""
    import ctypes
    import torch
    from mpm_b200 import _lib
    n = scene.n
    es = np.dtype(dtype).itemsize
    ctype = ctypes.c_double if es == 8 else ctypes.c_float
    ptrs = []
    for k in range(6):
        p = ctypes.c_void_p()
        _lib.check(_lib.lib().mpm_host_alloc(n * es, ctypes.byref(p)))
        arr = np.ctypeslib.as_array((ctype * n).from_address(p.value))
        arr[:] = (scene.x[:, k] if k < 3 else scene.v[:, k - 3])
        ptrs.append(p)
    io = _lib.MpmParticles(dtype=_lib.F64 if es == 8 else _lib.F32, x=ptrs[0], y=ptrs[1], z=ptrs[2], vx=ptrs[3],
                           vy=ptrs[4], vz=ptrs[5])
    sub = ctypes.c_int32()
    for _ in range(max(1, args.warmup)):
        _lib.check(_lib.lib().mpm_frame_host(sol.h, ctypes.byref(io), dt_req, 48, ctypes.byref(sub)), sol.h)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    sub_total = 0
    e0.record(ext)
    for _ in range(args.steps):
        _lib.check(_lib.lib().mpm_frame_host(sol.h, ctypes.byref(io), dt_req, 48, ctypes.byref(sub)), sol.h)
        sub_total += sub.value
    e1.record(ext)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    et = torch.tensor([ems, n * sub_total], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(et[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(et[1:2], op=dist.ReduceOp.SUM)
    for p in ptrs:
        _lib.lib().mpm_host_free(p)
    return {"value": float(et[1]) / (float(et[0]) / 1e3), "unit": UNIT,
            "h2d_bytes_per_step": 6 * es * n, "d2h_bytes_per_step": 6 * es * n,
            "ms_per_step": float(et[0]) / args.steps,
            "api": f"mpm_frame_host ({'f64' if es == 8 else 'f32'} pinned host arrays x, y, z, vx, vy, vz)"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    global np
    import numpy as np
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    if args.surrogate_only:
        if rank == 0:
            print(json.dumps({"surrogate": surrogate_leg(args.surrogate_steps),
                              "learned_return": learned_step_leg(args)}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.ensemble_only:
        out = ensemble_leg(args, rank, world, dist)
        if rank == 0:
            print(json.dumps({"ensemble": out}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.slabs and world > 1:
        slab_leg(args, rank, world, dist)
        dist.barrier()
        dist.destroy_process_group()
        return
    from mpm_b200 import _lib
    from mpm_b200.solver import Solver
    scene = make_scene(args)
    dt_req = scene.meta.get("dt", 2e-6)
    model = scene.materials[0].model
    sol = Solver(scene.domain, scene.n)
    sol.upload(scene)
    ext = torch.cuda.ExternalStream(sol.stream())
    clk = Clocks(local, args.clocks_csv)
    clk.__enter__()  # sampling starts before warm-up so the timed region is covered
    for _ in range(args.warmup):
        sol.step(dt_req)
    torch.cuda.synchronize()
    clk.wait_first_sample()
    if dist is not None:
        dist.barrier()
    # headline: the K requested steps through mpm_run (one call; the step boundaries are taken on
    # the device and the host synchronises once)
    launches0 = sol.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t_start = time.time()
    ev0.record(ext)
    substeps, _adv = sol.run(dt_req, args.steps)
    ev1.record(ext)
    torch.cuda.synchronize()
    t_end = time.time()
    launches = sol.launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    # the same K steps as K mpm_step calls (one host round trip each), for comparison
    pc0 = torch.cuda.Event(enable_timing=True)
    pc1 = torch.cuda.Event(enable_timing=True)
    pc_sub = 0
    pc0.record(ext)
    for _ in range(args.steps):
        pc_sub += sol.step(dt_req)[0]
    pc1.record(ext)
    torch.cuda.synchronize()
    per_call_ms = pc0.elapsed_time(pc1)
    # the same K steps again with a CUDA event pair around every kernel launch (on the library's
    # stream) for the per-kernel durations of the roofline; events between the launches of the
    # headline pass would add about 5% to it
    if dist is not None:
        dist.barrier()
    sol.profile(True)
    torch.cuda.synchronize()
    kp0 = torch.cuda.Event(enable_timing=True)
    kp1 = torch.cuda.Event(enable_timing=True)
    kp0.record(ext)
    prof_substeps, _ = sol.run(dt_req, args.steps)
    kp1.record(ext)
    torch.cuda.synchronize()
    t_end2 = time.time()
    prof = sol.profile_read()
    sol.profile(False)
    kernel_pass_ms = kp0.elapsed_time(kp1) / args.steps
    time.sleep(0.25)
    clk.__exit__()
    el_t = torch.tensor([ms, scene.n * substeps], dtype=torch.float64, device="cuda")
    if dist is not None:
        mx = el_t.clone()
        dist.all_reduce(mx[0:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(mx[1:2], op=dist.ReduceOp.SUM)
        el_t = mx
    ms_all, psteps = float(el_t[0]), float(el_t[1])
    value = psteps / (ms_all / 1e3)
    # roofline of the dominant kernel (g2p2g): algorithmic bytes per launch / average launch time
    dims, _ = sol.grid_dims()
    gm, _gp = sol.grid_debug(dt_req / 4)
    active_nodes = int(np.count_nonzero(gm > 0))
    g_ms, g_n = prof["g2p2g"]
    alg_bytes = scene.n * BYTES_PER_PARTICLE[model] + BYTES_PER_NODE * active_nodes
    hbm, peak_kind = peaks()
    # launches of the profile pass past the call's last substep return at once (the call launches
    # its substep estimate); their few microseconds stay in g_ms, but only the substeps that ran
    # count as launches, so the mean launch time is not understated
    ran = min(int(prof_substeps), int(g_n)) if g_n else 0
    launch_ms = g_ms / ran if ran else None
    achieved = alg_bytes / (launch_ms / 1e3) / 1e9 if launch_ms else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm if achieved else None,
                "traffic": TRAFFIC_PER_PARTICLE * scene.n, "traffic_source": TRAFFIC_SOURCE,
                "kernel": "k_g2p2g", "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": launch_ms,
                "launches_profiled": int(g_n), "substeps_ran": int(prof_substeps),
                "share_of_step": g_ms / sum(v[0] for v in prof.values()) if g_n else None,
                "timing": f"CUDA events around each launch in a second pass of the same {args.steps} steps "
                          f"({kernel_pass_ms:.3f} ms per step with the events)",
                "clocks": clk.summary(t_end, t_end2)}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": scene.meta["workload"], "particles": scene.n, "grid_nodes": list(dims),
                       "dt_requested": dt_req, "substeps_per_step": substeps / args.steps,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": f"particle state {scene.n * 160 / 1e6:.0f} MB > 126 MB L2 (no flush)",
                       "active_nodes": active_nodes,
                       "api": "mpm_run (all requested steps in one call)"},
            "roofline": roofline, "gpu_launches": launches,
            "step_per_call": {"value": scene.n * pc_sub / (per_call_ms / 1e3), "ms_per_step": per_call_ms / args.steps,
                              "api": "mpm_step once per requested step (a host round trip each)"},
            "kernel_ms": {k: v[0] for k, v in prof.items()}, "clocks": clk.summary(t_start, t_end)}
    # end to end through the C ABI with pinned host buffers (x, v in and out every step): FP64, the
    # type of the reference's particle arrays (Simulation3's Float64Arrays), is the headline; FP32
    # arrays are reported beside it
    if not args.no_e2e:
        line["e2e"] = e2e_leg(args, sol, scene, dt_req, ext, dist, np.float64)
        line["e2e_f32"] = e2e_leg(args, sol, scene, dt_req, ext, dist, np.float32)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        isa = orc.use_native()
        sample = sample_scene(scene, 2)
        threads = os.cpu_count() or 1
        rate, el, done, subs = cpu_oracle_rate(sample, dt_req, 50, threads, budget_s=20.0)
        rate1, el1, done1, subs1 = cpu_oracle_rate(sample, dt_req, 2, 1, budget_s=5.0)  # one worker thread
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "isa": isa,
                                "value_1_thread": rate1,
                                "sample": f"{sample.n}-particle sub-block (1/8) of the workload: {done} requested "
                                          f"steps of {dt_req} s ({subs} CFL substeps, {el:.1f} s) on {threads} "
                                          f"threads and {done1} ({subs1} substeps, {el1:.1f} s) on one; FP64 oracle "
                                          f"built {isa} with OpenMP"}
    if not args.no_ensemble:
        line["ensemble"] = ensemble_leg(args, rank, world, dist)
    if rank == 0 and world == 1 and not args.no_surrogate:
        line["surrogate"] = surrogate_leg(args.surrogate_steps)
        line["learned_return"] = learned_step_leg(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    sol.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
