"""CPU-only checks of the C-ABI library: it loads, exports every entry point
include/lhi.h declares, and its host-side scene code (boundary SDF, seeded
generator, the reference's lattice spawner) matches the oracle and the
reference's own fixture.  No compute call needs a GPU here."""
import ctypes as C
import hashlib
import json
import os
import re

import numpy as np

from liquidhairinteration_b200 import abi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def declared_entry_points():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"LHI_API\s+[\w\s\*]+?\b(lhi_\w+)\s*\(", text)
    return names


def test_library_exports_every_declared_symbol(lhi):
    names = declared_entry_points()
    assert len(names) >= 39
    L = lhi.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) <= set(lhi.SIGNATURES), set(names) - set(lhi.SIGNATURES)


def test_abi_struct_layouts():
    # sizes of the POD structs in include/lhi.h (x86-64 System V)
    assert C.sizeof(abi.GridDesc) == 64
    assert C.sizeof(abi.SolverParams) == 80
    assert C.sizeof(abi.LiquidParams) == 56
    assert C.sizeof(abi.SolveStats) == 40
    assert C.sizeof(abi.BoundaryNode) == 64
    assert C.sizeof(abi.FluidPrim) == 80
    assert C.sizeof(abi.RenderParams) == 20


def test_spawn_lattice_matches_liquiddata_frame0(lhi):
    """The reference's fixture LiquidData.csv frame 0 is SpawnParticles on
    Config/PureLiquid3D.json: [-1,1]^3, 64^3, 5000 particles, radius 2dx."""
    from liquidhairinteration_b200.model import spawn_lattice
    gold = json.load(open(os.path.join(GOLDEN, "liquiddata_frame0.json")))
    mn = np.array([-1, -1, -1], np.float32)
    mx = np.array([1, 1, 1], np.float32)
    dx = np.float32((mx[0] - mn[0]) / np.float32(64))
    off = np.float32(0.3) * (mx - mn)
    pos = spawn_lattice((mn + off).astype(np.float64), (mx - off).astype(np.float64), float(np.float32(2) * dx), 5000)
    assert pos.shape[0] == gold["count"]
    toks = ["%.6g" % float(v) for v in pos.reshape(-1)]
    assert len(toks) == gold["n_tokens"]
    assert toks[:300] == gold["head"]
    assert hashlib.sha256(",".join(toks).encode()).hexdigest() == gold["sha256"]


def test_boundary_eval_matches_oracle(lhi, oracle_mod):
    from liquidhairinteration_b200.model import OperatorBoundary, RectBoundary
    big = scenes.dam256()
    rng = np.random.default_rng(1)
    pts = rng.uniform(-0.2, 1.2, size=(20000, 3))
    for prec, dbl in (("fp32", False), ("fp64", True)):
        dt = np.float64 if dbl else np.float32
        out = np.empty(pts.shape[0], dt)
        arr = abi.boundary_array(big.boundary)
        p = np.ascontiguousarray(pts, dtype=dt)
        lhi.call("lhi_boundary_eval", arr, len(big.boundary), 0, abi.PRECISION_FP64 if dbl else abi.PRECISION_FP32,
                 p.ctypes.data_as(C.c_void_p), p.shape[0], out.ctypes.data_as(C.c_void_p))
        ref = oracle_mod.boundary_eval(big.boundary, pts, dbl)
        assert np.array_equal(out.view(np.uint64 if dbl else np.uint32), ref.view(np.uint64 if dbl else np.uint32))
    # the Python boundary classes build the same tree
    b = OperatorBoundary("Substract", RectBoundary((0.5, 0.5, 0.5), (0.4, 0.4, 0.4), True),
                         RectBoundary((0.5, 0.2, 0.5), (0.1, 0.1, 0.1)))
    a = b.Compute(pts)
    ref = oracle_mod.boundary_eval(b.nodes(), pts, False)
    assert np.array_equal(a, ref)


def test_seed_generator_deterministic_and_in_primitives(lhi):
    spec = scenes.dam(32)
    p1, v1 = scenes.seed(spec, "fp32")
    p2, v2 = scenes.seed(spec, "fp32")
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)
    assert p1.shape[0] % 8 == 0 and p1.shape[0] == scenes.particle_count(spec)
    assert (p1[:, 0] >= spec.dx).all() and (p1[:, 0] < 0.4 + spec.dx).all()
    assert (p1[:, 1] >= spec.dx).all() and (p1[:, 2] <= 1 - spec.dx).all()
    # 8 particles per cell, jitter +-0.25 sub-cell: each stays in its cell
    cells = np.floor(p1 / spec.dx).astype(int)
    assert (np.unique(cells.reshape(-1, 8, 3), axis=1).shape[1] == 1)
    d64, _ = scenes.seed(spec, "fp64")
    assert np.array_equal(d64.astype(np.float32), p1)
    # sphere primitive carries its own velocity
    s = scenes.dam128()
    s.n = 32
    s.boundary = [{"kind": abi.BOUNDARY_NONE, "left": 1}, scenes.walls(32)]
    p, v = scenes.seed(s, "fp32")
    moving = (v[:, 1] == -1.0)
    assert moving.any() and (np.linalg.norm(p[moving] - [0.7, 0.7, 0.5], axis=1) < 0.15 + 0.5 / 32).all()


def test_create_without_gpu_fails_loudly(lhi):
    """No CPU fallback: on a machine without a usable GPU, creating a handle
    returns a CUDA error instead of computing anywhere else."""
    import torch
    if torch.cuda.is_available():
        return
    L = lhi.lib()
    spec = scenes.dam(8)
    h = C.c_void_p()
    rc = L.lhi_liquid_create(C.byref(spec.grid_desc()), C.byref(spec.solver_params()),
                             C.byref(spec.liquid_params()), 0, C.byref(h))
    assert rc in (abi.LHI_E_CUDA, abi.LHI_E_OOM)
    assert not h.value
