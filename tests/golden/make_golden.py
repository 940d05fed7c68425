"""Regenerates the golden fixtures in this directory (run in a checkout that
has the reference tree at /root/reference and oracle/_ref/libref.so built).

* liquiddata_frame0.json : the reference's own fixture LiquidData.csv, frame 0
  (the SpawnParticles lattice of Config/PureLiquid3D.json): particle count,
  token count, SHA-256 of the comma-joined tokens and the first 300 tokens.
* ref_dam16.npz : outputs of the reference's own liquid step (its sources
  compiled from the reference tree, one OpenMP thread) on the 16^3 dam-break
  scene of liquidhairinteration_b200.scenes with walls three cells thick (the
  reference's own PCG diverges once fluid reaches the domain's outer cell
  layer, which one-cell walls allow): every stage of step 1, the solver
  matrix of every level, and positions after 3 steps.

    OMP_NUM_THREADS=1 python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from liquidhairinteration_b200 import abi, scenes  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

# the reference source tree, where this machine has one (LHI_REFERENCE_TREE overrides)
REFERENCE_TREE = os.environ.get("LHI_REFERENCE_TREE", "/root/reference")

# solver settings of the fixture run: the reference's own PCG and stopping rule
DAM16_SOLVER = dict(robust=False, max_iterations=100, tolerance=1e-4, num_level=4, num_pre_smooth=5,
                    num_post_smooth=5, num_final_smooth=20, smoothing_factor=0.5)


def dam16_spec():
    return scenes.dam(16, wall_cells=3)


def frame0():
    with open(os.path.join(REFERENCE_TREE, "LiquidData.csv")) as f:
        count = int(f.readline())
        line = f.readline()
    toks = [t for t in line.strip().split(",") if t]
    out = {"count": count, "n_tokens": len(toks),
           "sha256": hashlib.sha256(",".join(toks).encode()).hexdigest(), "head": toks[:300]}
    with open(os.path.join(HERE, "liquiddata_frame0.json"), "w") as f:
        json.dump(out, f)


def dam16():
    spec = dam16_spec()
    solver = spec.solver_params(**DAM16_SOLVER)
    cfg = spec.config_json(solver)
    ref = po.Reference(cfg)
    ref.set_boundary(spec.boundary)
    pos, vel = scenes.seed(spec, "fp32")
    ref.set_particles(pos, vel)
    dt = np.float32(spec.dt)
    out = {"pos0": pos, "vel0": vel, "solidPhi": ref.field("solidPhi"), "liquidWx": ref.field("liquidWx"),
           "liquidWy": ref.field("liquidWy"), "liquidWz": ref.field("liquidWz")}
    ref.pre_step(dt)
    out["liquidPhi"] = ref.field("liquidPhi")
    ref.particle_to_grid()
    for k in ("vx", "vy", "vz", "wx", "wy", "wz"):
        out["p2g_" + k] = ref.field(k)
    ref.apply_gravity(dt)
    out["grav_vy"] = ref.field("vy")
    ref.solve_pressure(dt)
    out["pressure"] = ref.field("pressure")
    out["rhs"] = ref.field("rhs")
    for lvl in range(4):
        out[f"Adiag{lvl}"] = ref.field("Adiag", lvl)
        out[f"Acoef{lvl}"] = ref.field("Acoef", lvl)
    for k in ("vx", "vy", "vz"):
        out["proj_" + k] = ref.field(k)
    ref.extrapolate()
    for k in ("vx", "vy", "vz"):
        out["ext_" + k] = ref.field(k)
    out["isValid"] = ref.field("isValid")
    ref.grid_to_particle()
    _, v1, a1 = ref.get_particles()
    out["g2p_vel"], out["g2p_aff"] = v1, a1
    ref.advect_particles(dt)
    out["pos1"] = ref.get_particles()[0]
    for _ in range(2):
        ref.pre_step(dt)
        ref.step(dt)
    out["pos3"] = ref.get_particles()[0]
    np.savez_compressed(os.path.join(HERE, "ref_dam16.npz"), **out)


if __name__ == "__main__":
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    frame0()
    dam16()
    print("golden fixtures written to", HERE)
