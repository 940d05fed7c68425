"""Trains the learned preconditioner on residuals that the plain GPU MGPCG
produces, then compares it with MGPCG and unpreconditioned CG.

    python -m liquidhairinteration_b200.train --out weights.lhinet [options]

Data: scenes of the batched form (scenes.random_scene: grid sizes,
fluid primitives and solid boxes drawn from the seed), each advanced a few
liquid steps on the GPU; the pressure solve of the last step records the
residual handed to the preconditioner at every PCG iteration.  Training
runs on the GPU (lhi_net_train: BF16 tcgen05 convolutions, FP32 Adam) with
the loss ||A M(r) - r||^2 / ||r||^2, cycling over the scenes.  The network is
fully convolutional, so weights trained on small grids apply to any grid.
"""
import argparse
import json
import time

import numpy as np

from . import abi, scenes
from ._lib import lib
from .net import LearnedNet


def record_scene(spec, warm_steps, snapshots):
    """A GPU model of ``spec`` advanced ``warm_steps`` steps whose last
    pressure solve recorded its residuals."""
    solver = spec.solver_params(coarse_cells=64)
    m = scenes.build(spec, "mixed", solver)
    for _ in range(warm_steps - 1):
        m.PreStep(spec.dt)
        m.Step(spec.dt)
    m.GetSolver().RecordResiduals(snapshots)
    m.PreStep(spec.dt)
    m.Step(spec.dt)
    return m


def record_on_policy(spec, net, warm_steps, snapshots, iterations=40):
    """A GPU model of ``spec``, advanced ``warm_steps - 1`` steps (FPCG with
    the V-cycle fallback), whose next pressure solve runs FPCG with the
    network alone (no fallback, ``iterations`` at most) and records the
    residuals that FPCG hands to the network."""
    learned = spec.solver_params(coarse_cells=64, preconditioner=abi.PRECOND_LEARNED)
    m = scenes.build(spec, "mixed", learned)
    s = m.GetSolver()
    s.SetNetwork(net, fallbackIterations=0)
    for _ in range(warm_steps - 1):
        m.PreStep(spec.dt)
        m.Step(spec.dt)
    s.SetNetwork(net, fallbackIterations=-1)
    s.RecordResiduals(snapshots)
    m.PreStep(spec.dt)
    m.Particle2Grid()
    m.ApplyGravity(spec.dt)
    # the recorded solve may stop at the iteration cap: only its residuals are kept
    lib().lhi_solver_solve(m._h, float(spec.density), float(spec.dt), None)
    return m


def compare(net, spec, warm_steps=2):
    """Iterations to ||r||/||b|| <= 1e-6 on one scene: FPCG with the network
    alone, FPCG with the V-cycle fallback, MGPCG, CG without preconditioner."""
    out = {}
    for name, over, fallback in (("fpcg_network_only", dict(preconditioner=abi.PRECOND_LEARNED), -1),
                                 ("fpcg", dict(preconditioner=abi.PRECOND_LEARNED), 0),
                                 ("mgpcg", dict(), None),
                                 ("cg", dict(preconditioner=abi.PRECOND_NONE), None)):
        solver = spec.solver_params(coarse_cells=64, max_iterations=2000, **over)
        m = scenes.build(spec, "mixed", solver)
        if fallback is not None:
            m.GetSolver().SetNetwork(net, fallbackIterations=fallback)
        for _ in range(warm_steps):
            m.PreStep(spec.dt)
            m.Step(spec.dt)
        st = m.GetSolver().Stats()
        out[name] = {"iterations": st["iterations"], "status": st["status"], "solve_ms": round(st["solve_ms"], 3)}
        if fallback is not None:
            out[name]["network_iterations"], out[name]["fallback_at"] = m.GetSolver().LearnedStats()
        m.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--scenes", type=int, default=16)
    ap.add_argument("--sizes", default="32,48,64")
    ap.add_argument("--warm-steps", type=int, default=3)
    ap.add_argument("--snapshots", type=int, default=64)
    ap.add_argument("--rounds", type=int, default=6)
    ap.add_argument("--steps", type=int, default=25, help="Adam steps per scene visit")
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--init", default=None, help="start from these weights")
    ap.add_argument("--eval", default="dam64")
    ap.add_argument("--budget-s", type=float, default=900.0)
    ap.add_argument("--on-policy", type=int, default=1, help="also train on residuals of FPCG with the network")
    ap.add_argument("--relu", type=int, default=0)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(a.seed)
    sizes = [int(s) for s in a.sizes.split(",")]
    t0 = time.time()
    net = LearnedNet(seed=a.seed)
    net.set_relu(bool(a.relu))
    if a.init:
        net.load(a.init)
    from ._lib import LhiError
    models = []
    while len(models) < a.scenes:
        spec = scenes.random_scene(rng, n=int(rng.choice(sizes)))
        try:
            m = record_scene(spec, a.warm_steps, a.snapshots)
        except LhiError as e:  # e.g. a closed fluid pocket without a free surface
            print(json.dumps({"skipped_scene": spec.n, "reason": str(e)}), flush=True)
            continue
        if m.GetSolver().NumSnapshots() == 0:
            m.close()
            continue
        m._spec = spec
        models.append(m)
    specs = [m._spec for m in models]
    log = []
    step = 0
    for rnd in range(a.rounds):
        # on-policy data: residuals of FPCG driven by the current network
        policy = []
        if a.on_policy and rnd > 0:
            for spec in specs:
                try:
                    policy.append(record_on_policy(spec, net, a.warm_steps, a.snapshots))
                except LhiError:
                    pass
        for k, m in enumerate(models + policy):
            if time.time() - t0 > a.budget_s:
                break
            first, last = net.train(m, a.steps, a.batch, a.lr, seed=a.seed * 100003 + step)
            step += a.steps
            log.append({"round": rnd, "scene": k, "adam_steps": step, "loss_first": first, "loss_last": last})
        for m in policy:
            m.close()
        print(json.dumps(log[-1]), flush=True)
    for m in models:
        m.close()
    net.save(a.out)
    result = {"adam_steps": step, "scenes": a.scenes, "batch": a.batch, "lr": a.lr, "train_s": round(time.time() - t0, 1),
              "final_loss": log[-1]["loss_last"] if log else None,
              "eval": {a.eval: compare(net, scenes.get(a.eval))}}
    print(json.dumps(result), flush=True)
    net.close()
    return result


if __name__ == "__main__":
    main()
