"""Benchmark of the liquid step: ms/step of the 256^3 dam break on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm: the scene lives on the GPU; W untimed steps, then K timed steps
(PreStep + Step: sort, liquid SDF, P2G, gravity, pressure solve to
||r||/||b|| <= 1e-6 on the true residual, velocity update, extrapolation, G2P,
advection) bracketed by a barrier and synchronisation, timed with CUDA events
on the library's stream, max over ranks.  Under torchrun every rank runs an
independent replica of the scene (replicas only: the step has no exchange).

e2e: the same step through the public C-ABI with host buffers: every step
uploads the particle state (position, velocity, affine) from pinned memory,
steps, and downloads it again.

The reference arm (--impl reference) times the reference's own CPU code
(oracle/_ref/libref.so, its sources compiled from the reference tree) on
this very workload: the 256^3 scene with its 32M particles, one full
PreStep + Step per timed step, with the OpenMP thread count that a short
calibration on the 32^3 scene finds fastest.  It loads no CUDA library: the
particles come from the scene generator compiled into the oracle library.

error_vs_fp64_oracle (our arm, after every timed region): one projection of
the scene's current state on the GPU against the FP64 CPU oracle solved to
||r||/||b|| <= 1e-12 on the same float inputs.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "256³ ms/step, solve ms: learned-precond FPCG vs plain MGPCG, 1 B200, rr≤1e-6"
UNIT = "ms/step"

# The reference's PCG does not converge on this scene (once fluid reaches the
# domain's outer cell layer its update region and smoother break down), so the
# reference arm runs its solver for the iteration count our MGPCG needs on
# this workload.
REFERENCE_PCG_ITERATIONS = 21
# cpu_baseline of our arm: a bounded sample, the full reference step on the
# same scene at 32^3 (1/512 of the cells and particles), time x512.  Every
# reference loop is linear in cells or particles and the small grid is
# cache-resident, so the extrapolation favours the reference.
REFERENCE_SAMPLE_N = 32
PRECISION_TEXT = {
    "mixed": "FP32 V-cycle and loop SpMV, FP64 x, dots, finest-level matrix and right-hand side for the true "
             "residual every 10 iterations and the final check",
    "fp64": "all FP64", "fp32": "all FP32"}


def scene_text(spec):
    parts = []
    for p in spec.prims:
        if p["kind"] == 0:
            parts.append("block [%g,%g]x[%g,%g]x[%g,%g)" % (p["a"][0], p["b"][0], p["a"][1], p["b"][1], p["a"][2],
                                                             p["b"][2]))
        else:
            parts.append("sphere r=%g at (%g,%g,%g)" % (p["b"][0], *p["a"]))
    if spec.name == "dam256":
        parts.append("two solid boxes")
    return ", ".join(parts)


# the grid inputs of a pressure solve, shared by the GPU and the oracle check
GRID_INPUTS = ("vx", "vy", "vz", "liquidPhi", "liquidWx", "liquidWy", "liquidWz")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "replica-check"],
                    help="replica-check: the launcher and rank plumbing alone (gloo on CPU, no GPU work)")
    ap.add_argument("--scene", default="dam256")
    ap.add_argument("--precision", default="mixed", choices=["fp32", "mixed", "fp64"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--eager", action="store_true", help="host-driven PCG loop instead of the solve graph")
    ap.add_argument("--no-fpcg", action="store_true", help="skip the learned-preconditioner FPCG leg")
    ap.add_argument("--no-oracle-check", action="store_true", help="skip error_vs_fp64_oracle")
    ap.add_argument("--ref-steps", type=int, default=1,
                    help="reference arm: full-size reference steps timed (each takes minutes)")
    ap.add_argument("--ref-iterations", type=int, default=REFERENCE_PCG_ITERATIONS,
                    help="reference arm: PCG iterations per step (our MGPCG's count on the workload)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), int(
        os.environ.get("WORLD_SIZE", "1"))


def rank_reducers(world, device):
    """barrier() and max_over_ranks(v) over this run's process group (both
    plain pass-throughs for one rank).  Every timed number of a multi-replica
    run is the maximum over ranks."""
    import torch

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    return barrier, max_over_ranks


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        import statistics
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "", 1).isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, n in enumerate(names):
                if s[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ------------------------------------------------------------------ peaks
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# Algorithmic bytes per launch of each timed category: A = active cells of
# level 0 (active tiles x 2048 cells), C = all cells, P = particles, s =
# bytes per scalar.
def algorithmic_bytes(cat, A, C_cells, P, scalar=4):
    s = scalar
    table = {
        # one red-black sweep (both colours) on level 0 over the active
        # tiles: z, r, diag, 3 face coefficients and the neighbour mask read
        # once, z written once
        "smooth_fine": (7 * s + 1) * A,
        # Ap = A p and p.Ap: p, diag, 3 face coefficients, mask read, Ap written
        "spmv": (5 * s + 1 + s) * A,
        # P2G accumulation (k_p2g; the normalisation is timed with "grid"):
        # position, velocity, affine read once per particle, w and v written
        # once per face of the three components
        "p2g": 15 * s * P + 6 * s * C_cells,
        # G2P + advection: position read, velocity/affine/position written,
        # cell key and index written, face velocities read once; the sort's
        # deferred permutation: its index and the id read, the id written
        "g2p": (3 + 15) * s * P + 8 * P + 12 * P + 3 * s * C_cells,
    }
    return table.get(cat)


# --------------------------------------------------------------- our arm
def run_ours(args):
    import numpy as np
    import torch
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local_rank))
    from liquidhairinteration_b200 import scenes
    from liquidhairinteration_b200.model import kernel_launch_count

    spec = scenes.get(args.scene)
    solver = spec.solver_params(eager=1 if args.eager else 0)
    model = scenes.build(spec, args.precision, solver)
    ps = model.GetParticleSystem()
    n_particles = ps.NumParticles()
    stream = torch.cuda.ExternalStream(model.stream_ptr())

    barrier, max_over_ranks = rank_reducers(world, "cuda")

    for _ in range(args.warmup):
        model.PreStep(spec.dt)
        model.Step(spec.dt)
    model.sync()

    # ---- timed region: K steps on device-resident state (the solve runs as
    # one CUDA graph per step; no per-kernel events in here)
    clocks = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local_rank)
    iters, solve_ms = [], []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    model.sync()
    launches0 = kernel_launch_count()
    clocks.start()
    ev0.record(stream)
    for _ in range(args.steps):
        model.PreStep(spec.dt)
        model.Step(spec.dt)
        st = model.GetSolver().Stats()
        iters.append(st["iterations"])
        solve_ms.append(st["solve_ms"])
    ev1.record(stream)
    ev1.synchronize()
    launches = kernel_launch_count() - launches0
    clock_info = clocks.stop()
    torch.cuda.synchronize()
    barrier()
    ms_step = max_over_ranks(ev0.elapsed_time(ev1) / args.steps)
    solve_avg = max_over_ranks(sum(solve_ms) / len(solve_ms))

    # ---- per-kernel breakdown: separate profiled steps (CUDA events around
    # every launch on the library's stream; the PCG loop runs host-driven
    # here, which changes launch gaps but not kernel durations)
    prof_steps = max(1, min(3, args.steps))
    model.profile(True)
    for _ in range(prof_steps):
        model.PreStep(spec.dt)
        model.Step(spec.dt)
    model.profile(False)
    prof = model.profile_read()
    active, total, _ = model.GetSolver().ActiveTiles(0)
    active_cells = active * 8 * 8 * 32

    # ---- roofline of the dominant kernel category
    peak, peak_kind = measured_peaks()
    cells = spec.n ** 3
    scalar = 8 if args.precision == "fp64" else 4
    dominant = max((k for k in prof if algorithmic_bytes(k, active_cells, cells, n_particles, scalar) is not None),
                   key=lambda k: prof[k][1])
    n_launch, tot_ms = prof[dominant]
    algo = algorithmic_bytes(dominant, active_cells, cells, n_particles, scalar)
    avg_ms = tot_ms / max(n_launch, 1)
    achieved = algo / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if os.path.exists(tpath):
        tj = json.load(open(tpath))
        tv = tj.get(args.scene, {}).get(dominant)
        if isinstance(tv, dict):  # measured at another active-tile count of the scene: scaled by active tiles
            traffic = int(round(tv["bytes_per_launch"] * active / max(tv["active_tiles"], 1)))
        else:
            traffic = tv
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": int(algo), "avg_launch_ms": round(avg_ms, 5),
                "launches_profiled": n_launch, "active_tiles_level0": f"{active}/{total}"}
    # every category with a per-launch byte model, the stencil kernels among them
    per_kernel = {}
    for k in sorted(prof):
        b = algorithmic_bytes(k, active_cells, cells, n_particles, scalar)
        nl, ms = prof[k]
        if b is None or nl == 0 or ms <= 0:
            continue
        gbs = b / (ms / nl * 1e-3) / 1e9
        per_kernel[k] = {"achieved": round(gbs, 1), "frac": round(gbs / peak, 4), "avg_launch_ms": round(ms / nl, 5),
                         "algorithmic_bytes_per_launch": int(b)}
    roofline["kernels"] = per_kernel
    # the whole step against HBM: the byte model of liquidhairinteration_b200/roofline.py over the
    # timed steps' mean iteration count
    from liquidhairinteration_b200 import roofline as step_model
    sb = step_model.step_bytes(n_particles, cells, active_cells, float(sum(iters)) / len(iters), scalar)
    roofline["step"] = {"algorithmic_bytes": int(sb), "achieved": round(sb / (ms_step * 1e-3) / 1e9, 1),
                        "frac": round(sb / (ms_step * 1e-3) / 1e9 / peak, 4),
                        "what": "whole step: algorithmic bytes of every stage (roofline.step_bytes) / ms_per_step"}

    # ---- learned-preconditioner FPCG on the same scene (V-cycle fallback on
    # a < 5% residual drop), timed the same way over a few steps
    fpcg = None
    if not args.no_fpcg:
        fpcg = run_fpcg(args, spec, stream_of=lambda m: torch.cuda.ExternalStream(m.stream_ptr()))

    # ---- e2e through the C-ABI with host buffers
    e2e = None
    if not args.no_e2e:
        dt_np = np.float64 if args.precision == "fp64" else np.float32
        pos, vel, aff = ps.GetParticles()
        hp = [torch.from_numpy(a.copy()).pin_memory() for a in (pos, vel, aff)]
        host = [t.numpy() for t in hp]
        for _ in range(1):
            ps.SetParticles(*host)
            model.PreStep(spec.dt)
            model.Step(spec.dt)
            p2, v2, a2 = ps.GetParticles()
        lib = model  # noqa
        from liquidhairinteration_b200._lib import call
        ptrs = [h.ctypes.data_as(C.c_void_p) for h in host]
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            call("lhi_liquid_set_particles", model._h, n_particles, ptrs[0], ptrs[1], ptrs[2])
            model.PreStep(spec.dt)
            model.Step(spec.dt)
            call("lhi_liquid_get_particles", model._h, ptrs[0], ptrs[1], ptrs[2])
        e1.record(stream)
        e1.synchronize()
        barrier()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
        nbytes = n_particles * 15 * np.dtype(dt_np).itemsize
        e2e = {"value": round(e2e_ms, 3), "unit": UNIT, "h2d_bytes_per_step": int(nbytes),
               "d2h_bytes_per_step": int(nbytes)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(spec)

    # ---- the checker, after every timed region: one projection against the
    # FP64 oracle (rank 0 of a single-replica run)
    check = None
    if rank == 0 and world == 1 and not args.no_oracle_check:
        check = oracle_check(model, spec)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(ms_step, 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else
            {"fp32": "f32", "fp64": "f64"}[args.precision], "data": "synthetic",
            "config": {
                "workload": f"{spec.name}: {spec.n}^3 unit-cube dam break ({scene_text(spec)}), {n_particles} "
                            f"particles (8 per cell, seed {spec.seed}), dt {spec.dt:.6g}, one replica per GPU",
                "solver": f"MGPCG: {solver.num_level} levels, {solver.num_pre_smooth}+{solver.num_post_smooth} "
                          f"red-black damped Gauss-Seidel (w={solver.smoothing_factor:g}), {solver.num_final_smooth} coarsest sweeps, flexible "
                          "CG on every fluid cell, " + PRECISION_TEXT[args.precision] +
                          ", ||r||/||b|| <= 1e-6 on the true residual",
                "precision": args.precision,
                "l2": "inputs larger than L2 (grid fields ~1.2 GB, particles ~1.9 GB)",
                "parallelism": f"replicas x{world}",
            },
            "solve_ms": round(solve_avg, 3), "cg_iterations": round(sum(iters) / len(iters), 2),
            "particles_per_s": round(n_particles / (ms_step * 1e-3), 1),
            "scenes_per_s": round(world * 1000.0 / ms_step, 3),
            "fpcg": fpcg,
            "error_vs_fp64_oracle": check,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clock_info,
            "kernel_ms_per_step": {k: round(v[1] / prof_steps, 3) for k, v in prof.items()},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_fpcg(args, spec, stream_of, steps=None):
    """ms/step, solve ms and iterations of FPCG with the shipped network
    (liquidhairinteration_b200/weights/fpcg.lhinet) on the same scene."""
    import torch
    from liquidhairinteration_b200 import abi, scenes
    from liquidhairinteration_b200.net import LearnedNet
    if args.precision == "fp64":
        return {"unavailable": "the learned preconditioner runs on FP32 / mixed handles"}
    net = LearnedNet(seed=0)
    net.load(os.path.join(ROOT, "liquidhairinteration_b200", "weights", "fpcg.lhinet"))
    m = scenes.build(spec, args.precision, spec.solver_params(preconditioner=abi.PRECOND_LEARNED))
    m.GetSolver().SetNetwork(net, fallbackIterations=0)
    k = steps or max(1, min(5, args.steps))
    for _ in range(max(1, min(2, args.warmup))):
        m.PreStep(spec.dt)
        m.Step(spec.dt)
    stream = stream_of(m)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    it, sol, nit, fb = [], [], [], []
    m.sync()
    e0.record(stream)
    for _ in range(k):
        m.PreStep(spec.dt)
        m.Step(spec.dt)
        st = m.GetSolver().Stats()
        it.append(st["iterations"])
        sol.append(st["solve_ms"])
        a, b = m.GetSolver().LearnedStats()
        nit.append(a)
        fb.append(b)
    e1.record(stream)
    e1.synchronize()
    out = {"ms_per_step": round(e0.elapsed_time(e1) / k, 3), "solve_ms": round(sum(sol) / k, 3),
           "cg_iterations": round(sum(it) / k, 2), "network_iterations": round(sum(nit) / k, 2),
           "fallback_at": fb, "steps": k,
           "network": "3-level conv net, 16/32/64 channels, BF16 tcgen05 convolutions, liquidhairinteration_b200/weights/fpcg.lhinet"}
    m.close()
    net.close()
    return out


# ------------------------------------------------------------- checker
def oracle_check(model, spec):
    """Error of one projection against the FP64 oracle.

    From the model's current state (after the timed steps): PreStep, P2G and
    gravity on the GPU; the GPU's float grid inputs then go to both the GPU
    projection (the handle's own precision and stopping rule) and the FP64
    CPU oracle, which solves the same system to ||r||/||b|| <= 1e-12
    (CGSolver<3>::Solve, PressureSolver.cpp:839-934) and applies the same
    velocity update.  Reports the pressure's relative L2 error and the
    post-projection divergence max-norm of both (LiquidModel.cpp:1066-1083,
    max-norm over the cells whose six faces the update touches)."""
    import numpy as np
    from oracle import pyoracle as po
    po.set_threads(0)
    t0 = time.perf_counter()
    dt = spec.dt
    model.PreStep(dt)
    model.Particle2Grid()
    model.ApplyGravity(dt)
    fields = {f: model.field(f) for f in GRID_INPUTS}
    div_before = model.ComputeDivergenceMax()
    model.Projection(dt)
    st = model.GetSolver().Stats()
    p_gpu = model.field("pressure").astype(np.float64)
    div_gpu = model.ComputeDivergenceMax()
    o = po.Oracle(spec.grid_desc(), spec.solver_params(tolerance=1e-12, max_iterations=400), spec.liquid_params(),
                  dbl=True)
    o.set_boundary(spec.boundary)
    for f, v in fields.items():
        o.set_field(f, v.astype(np.float64))
    st_o = o.solve(spec.density, dt)  # the oracle holds no particles: solve + velocity update by hand
    o.velocity_update(dt)
    p_o = o.field("pressure")
    _, div_o = o.divergence()
    nrm = float(np.linalg.norm(p_o))
    rel = float(np.linalg.norm(p_gpu - p_o) / (nrm if nrm > 0 else 1.0))
    return {"pressure_rel_l2": rel, "pressure_tolerance": 1e-5,
            "gpu_true_residual_rel": st["true_residual"] / st["initial_residual"] if st["initial_residual"] else 0.0,
            "gpu_iterations": st["iterations"], "oracle_iterations": st_o["iterations"],
            "oracle_rel_residual": st_o["true_residual"] / st_o["initial_residual"] if st_o["initial_residual"] else 0.0,
            "div_max_before": div_before, "div_max_after_gpu": div_gpu, "div_max_after_oracle": div_o,
            "oracle_threads": po.get_threads(), "check_s": round(time.perf_counter() - t0, 1),
            "what": "one projection of the scene's state after the timed steps; the same float inputs; oracle FP64 "
                    "solved to 1e-12; positions: tests/test_gpu_configs.py (64^3, 100 FP64 steps)"}


# --------------------------------------------------------- reference arm
def reference_model(po, spec, iterations):
    """The reference's LiquidModel<3> on the scene (Scene<3> built from the
    reference JSON schema), PCG capped at ``iterations``."""
    # the scene's own MG settings (levels, sweeps) with the reference's solver semantics
    solver = spec.solver_params(robust=False, max_iterations=iterations, tolerance=1e-30)
    ref = po.Reference(spec.config_json(solver))
    ref.set_boundary(spec.boundary)
    return ref


def scaled_scene(n):
    """dam256's layout (block, walls one cell thick, the two solid boxes) on an n^3 grid."""
    from liquidhairinteration_b200 import scenes
    small = scenes.dam256()
    small.n = n
    small.boundary = [dict(small.boundary[0]), scenes.walls(n)] + [dict(b) for b in small.boundary[2:]]
    return small


def reference_stepper(po, spec, iterations=REFERENCE_PCG_ITERATIONS):
    """A function that times one reference PreStep + Step on the scene and
    returns seconds, and the particle count.  Each timed step restarts from
    the seeded state so the reference's own (non-converging) PCG cannot
    accumulate NaN from step to step."""
    import numpy as np
    pos, vel = po.seed_scene(spec, "fp32")
    ref = reference_model(po, spec, iterations)
    dt = np.float32(spec.dt)

    def step():
        ref.set_particles(pos, vel)
        t = time.perf_counter()
        ref.pre_step(dt)
        ref.step(dt)
        return time.perf_counter() - t

    return step, pos.shape[0]


def fastest_reference_threads(po, spec):
    """OpenMP thread count with the fastest reference step on the scene's
    layout at 32^3.  The reference's ComputeLiquidPhi takes an omp critical
    section per (particle, cell) pair (LiquidModel.cpp:540-560), so more
    threads can make it slower; the arm gives the reference its best count."""
    cores = os.cpu_count() or 1
    cands = sorted({c for c in (1, 2, 4, 8, 16, 32, 64, cores) if c <= cores})
    step, _ = reference_stepper(po, scaled_scene(REFERENCE_SAMPLE_N))
    times = {}
    for c in cands:
        po.set_reference_threads(c)
        step()
        times[c] = min(step() for _ in range(2))
    best = min(times, key=times.get)
    return best, {str(c): round(t * 1e3, 1) for c, t in times.items()}


def cpu_baseline(spec, steps=3):
    from oracle import pyoracle as po
    if not po.reference_available():
        return None
    cores = os.cpu_count() or 1
    po.set_reference_threads(cores)
    step, npart = reference_stepper(po, scaled_scene(REFERENCE_SAMPLE_N))
    step()  # warm-up
    secs = [step() for _ in range(steps)]
    scale = (spec.n / REFERENCE_SAMPLE_N) ** 3
    ms = sum(secs) / len(secs) * 1e3 * scale
    return {"value": round(ms, 1), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"bounded sample: reference LiquidModel<3>::PreStep+Step (OpenMP, {cores} threads) on the same "
                      f"scene layout at {REFERENCE_SAMPLE_N}^3 ({npart} particles), PCG capped at "
                      f"{REFERENCE_PCG_ITERATIONS} iterations, {steps} steps, time x{scale:.0f}; the full-size "
                      f"measurement is the --impl reference arm"}


def run_reference(args):
    """The reference's own CPU step on the full workload (see the module
    docstring).  Rank 0 alone runs it; the other ranks exit at once."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    from oracle import pyoracle as po
    from liquidhairinteration_b200 import scenes
    if not po.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref.so was not built"}))
        return
    spec = scenes.get(args.scene)
    t0 = time.perf_counter()
    threads, calib = fastest_reference_threads(po, spec)
    po.set_reference_threads(threads)
    step, npart = reference_stepper(po, spec, args.ref_iterations)
    setup_s = time.perf_counter() - t0
    k = max(1, args.ref_steps)
    secs = [step() for _ in range(k)]
    ms = sum(secs) / len(secs) * 1e3
    sample = (f"reference LiquidModel<3>::PreStep+Step (its own sources, OpenMP, {threads} threads: the fastest of a "
              f"32^3 calibration) on the full {spec.n}^3 scene, {npart} particles, PCG capped at "
              f"{args.ref_iterations} iterations (the GPU's count; the reference's own PCG does not converge on "
              f"this scene), {k} step(s) timed, no warm-up step (each takes minutes)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(ms, 1), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 1), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{spec.name}: the same {spec.n}^3 scene and particles as our arm (reference CPU path)",
                   "parallelism": f"OpenMP x{threads}"},
        "ref_steps_timed": k, "step_seconds": [round(s, 2) for s in secs], "setup_s": round(setup_s, 1),
        "thread_calibration_ms_at_32": calib,
        "cpu_baseline": {"value": round(ms, 1), "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(ms, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ------------------------------------------------------- replica launch
def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_replicas(n, argv, visible_gpus):
    """Runs this script as n ranks of one node under torch.distributed.run
    (one replica of the scene per GPU) and returns its exit code.  Fails
    loudly when fewer than n GPUs are visible."""
    if n > visible_gpus:
        print(f"bench.py: --gpus {n} needs {n} visible GPUs, {visible_gpus} found", file=sys.stderr, flush=True)
        return 2
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={_free_port()}", os.path.abspath(__file__)] + list(argv)
    return subprocess.call(cmd)


def run_replica_check(args):
    """Every rank joins a gloo group, takes the bench's barrier and
    max-over-ranks, and rank 0 prints the run's rank count and the maximum
    of the ranks' values (rank r contributes r + 1)."""
    import datetime
    import torch
    rank, _, world = dist_env()
    if world > 1:
        torch.distributed.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    barrier, max_over_ranks = rank_reducers(world, "cpu")
    barrier()
    v = max_over_ranks(float(rank + 1))
    barrier()
    if rank == 0:
        print(json.dumps({"impl": "replica-check", "n_ranks": world, "max_over_ranks": v}), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.impl != "reference" and args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # not under a launcher yet: start one rank per GPU
        if args.impl == "replica-check":
            visible = args.gpus
        else:
            import torch
            visible = torch.cuda.device_count()
        sys.exit(launch_replicas(args.gpus, sys.argv[1:], visible))
    if args.impl == "reference":
        run_reference(args)
    elif args.impl == "replica-check":
        run_replica_check(args)
    else:
        world = dist_env()[2]
        if world != args.gpus:
            print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE {world}", file=sys.stderr, flush=True)
            sys.exit(2)
        run_ours(args)


if __name__ == "__main__":
    main()
