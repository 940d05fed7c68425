"""The batched form: many independent scenes of uneven grid sizes stepped
together on one GPU.

Every scene is a handle in asynchronous mode (lhi_liquid_set_async) with its
own CUDA stream, and its pressure solve is one CUDA graph with the PCG loop
on the device, so one batch step enqueues every scene's whole liquid step
before the host waits once; the scenes' kernels run concurrently.  An
autotuner picks, per grid size, the smoother sweeps and the size below which
the coarse multigrid levels run in one CTA, by the time to solution it
measures on the first scene of that size.  Optionally every solve's
residuals, cell classes and solution are logged as FP32 training data.

    python -m liquidhairinteration_b200.batch --scenes 48 --steps 100 [--log-dir DIR]
"""
import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import abi, scenes
from ._lib import call

# candidate (pre = post sweeps, coarse-CTA cell limit) the autotuner tries
CANDIDATES = [(1, 512), (2, 512), (2, 4096), (3, 4096)]


def build_scene(spec, precision, pre, coarse, coarse_operator=abi.COARSE_GALERKIN):
    solver = spec.solver_params(num_pre_smooth=pre, num_post_smooth=pre, coarse_cells=coarse,
                                coarse_operator=coarse_operator)
    return scenes.build(spec, precision, solver)


def stats_of(m):
    st = abi.SolveStats()
    call("lhi_solver_get_stats", m._h, C.byref(st))
    return st.as_dict()


def autotune(spec, precision, steps=3, coarse_operator=abi.COARSE_GALERKIN):
    """(pre/post sweeps, coarse cells) with the smallest mean solve time on
    ``spec`` after one warm-up step."""
    best, table = None, {}
    for pre, coarse in CANDIDATES:
        m = build_scene(spec, precision, pre, coarse, coarse_operator)
        m.PreStep(spec.dt)
        m.Step(spec.dt)
        t = []
        for _ in range(steps):
            m.PreStep(spec.dt)
            m.Step(spec.dt)
            t.append(m.GetSolver().Stats()["solve_ms"])
        m.close()
        ms = float(np.mean(t))
        table[f"{pre}+{pre} sweeps, coarse<={coarse}"] = round(ms, 3)
        if best is None or ms < best[0]:
            best = (ms, pre, coarse)
    return (best[1], best[2]), table


class BatchRunner:
    def __init__(self, specs, precision="mixed", tune=True, log_dir=None, coarse_operator=abi.COARSE_GALERKIN):
        self.specs = specs
        self.precision = precision
        self.coarse_operator = coarse_operator
        self.tuned, self.tune_tables = {}, {}
        for spec in specs:
            if spec.n not in self.tuned:
                if tune:
                    self.tuned[spec.n], self.tune_tables[spec.n] = autotune(spec, precision,
                                                                             coarse_operator=coarse_operator)
                else:
                    self.tuned[spec.n] = (2, 4096)
        self.models = []
        for spec in specs:
            pre, coarse = self.tuned[spec.n]
            m = build_scene(spec, precision, pre, coarse, coarse_operator)
            if log_dir is None:
                call("lhi_liquid_set_async", m._h, 1)
            else:
                m.GetSolver().RecordResiduals(64)
            self.models.append(m)
        self.log_dir = log_dir
        self.logged = 0
        self.step_index = 0
        # a scene whose solve produced NaN/Inf is not stepped again (its
        # particles carry no meaning any more; stepping them only wastes time)
        self.alive = [True] * len(self.models)
        self.diverged = {}
        if log_dir:
            os.makedirs(log_dir, exist_ok=True)

    def step(self):
        """One liquid step of every live scene: all enqueued, then one wait.
        Returns the solve statistics of the scenes stepped."""
        from ._lib import LhiError
        live = [k for k, a in enumerate(self.alive) if a]
        self.last_live = live  # the scenes of the returned statistics, in order
        for k in live:
            try:
                self.models[k].PreStep(self.specs[k].dt)
                self.models[k].Step(self.specs[k].dt)
            except LhiError as e:  # synchronous mode reports a NaN solve here
                self.alive[k] = False
                self.diverged[k] = self.step_index
        out = []
        for k in live:
            if not self.alive[k]:
                out.append({"status": abi.LHI_E_NAN, "iterations": 0})
                continue
            st = stats_of(self.models[k])
            if st["status"] == abi.LHI_E_NAN:
                self.alive[k] = False
                self.diverged[k] = self.step_index
            out.append(st)
        if self.log_dir:
            self._log()
        self.step_index += 1
        return out

    def _log(self):
        """One FP32 shard per step: every scene's recorded residuals, cell
        classes (liquid SDF sign) and MGPCG solution."""
        shard = {}
        for k, m in enumerate(self.models):
            n = m.GetSolver().NumSnapshots()
            if n == 0:
                continue
            snaps = np.empty((n, m.field("pressure").size), np.float32)
            for i in range(n):
                call("lhi_solver_get_snapshot", m._h, i, snaps[i].ctypes.data_as(C.c_void_p))
            shard[f"r{k}"] = snaps
            shard[f"fluid{k}"] = (m.field("liquidPhi") <= 0).astype(np.uint8)
            shard[f"x{k}"] = m.field("pressure")
            shard[f"dims{k}"] = np.array([self.specs[k].n] * 3, np.int32)
            self.logged += n
            m.GetSolver().RecordResiduals(64)
        np.savez(os.path.join(self.log_dir, f"step{self.step_index:04d}.npz"), **shard)

    def close(self):
        for m in self.models:
            m.close()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=48)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--log-dir", default=None)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--coarse", default="galerkin", choices=["galerkin", "reference"],
                    help="coarse multigrid operators: Galerkin (default) or the reference's re-discretisation")
    a = ap.parse_args(argv)
    cop = abi.COARSE_GALERKIN if a.coarse == "galerkin" else abi.COARSE_REFERENCE
    rng = np.random.default_rng(a.seed)
    specs = [scenes.random_scene(rng) for _ in range(a.scenes)]
    t0 = time.time()
    runner = BatchRunner(specs, a.precision, tune=not a.no_tune, log_dir=a.log_dir, coarse_operator=cop)
    setup_s = time.time() - t0
    import torch
    torch.cuda.synchronize()
    t1 = time.time()
    bad, iters, scene_steps = 0, [], 0
    scene_iters, scene_n = np.zeros(len(specs)), np.zeros(len(specs))
    for _ in range(a.steps):
        st = runner.step()
        scene_steps += len(st)
        bad += sum(1 for s in st if s["status"] != abi.LHI_OK)
        iters.append(np.mean([s["iterations"] for s in st]) if st else 0.0)
        for k, s in zip(runner.last_live, st):
            scene_iters[k] += s["iterations"]
            scene_n[k] += 1
    wall = time.time() - t1
    cells = sum(s.n ** 3 for s in specs)
    # the batch against HBM: the step byte model (roofline.step_bytes) of every scene over its steps
    # (active cells of its finest level as after the last step)
    from . import roofline
    moved = 0.0
    for k, (spec, m) in enumerate(zip(specs, runner.models)):
        if scene_n[k] == 0:
            continue
        active = m.GetSolver().ActiveTiles(0)[0] * 8 * 8 * 32
        P = m.GetParticleSystem().NumParticles()
        s_b = 8 if a.precision == "fp64" else 4
        moved += scene_n[k] * (roofline.particle_bytes(P, s_b) + roofline.grid_bytes(spec.n ** 3, s_b))
        moved += roofline.solve_bytes(active, scene_iters[k], s_b)
    peak, peak_kind = roofline.hbm_peak()
    gbs = moved / wall / 1e9
    res = {"scenes": a.scenes, "steps": a.steps, "sizes": sorted({s.n for s in specs}),
           "cells": cells, "wall_s": round(wall, 3), "scene_steps_per_s": round(scene_steps / wall, 2),
           "ms_per_batch_step": round(1000 * wall / a.steps, 3), "mean_cg_iterations": round(float(np.mean(iters)), 2),
           "failed_solves": bad, "diverged_scenes": {str(k): v for k, v in runner.diverged.items()},
           "hbm": {"algorithmic_bytes_per_batch_step": int(moved / a.steps), "achieved_gbs": round(gbs, 1),
                   "frac": round(gbs / peak, 4), "peak_gbs": peak, "peak_kind": peak_kind,
                   "what": "every scene's step bytes (roofline.step_bytes) / wall time of the batch steps"},
           "coarse_operator": a.coarse,
           "setup_s": round(setup_s, 1),
           "autotuned": {str(k): {"sweeps": v[0], "coarse_cells": v[1]} for k, v in runner.tuned.items()},
           "autotune_solve_ms": {str(k): v for k, v in runner.tune_tables.items()},
           "snapshots_logged": runner.logged}
    runner.close()
    print(json.dumps(res), flush=True)
    return res


if __name__ == "__main__":
    main()
