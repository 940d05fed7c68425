"""The CPU oracle against the reference itself.

* the committed golden fixture (outputs of the reference's own sources run
  with one OpenMP thread, tests/golden/make_golden.py), bit for bit;
* the reference cross-check build, live, where it is available here;
* the solver findings the scenes rely on.
"""
import json
import os

import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import assert_bitwise

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _golden_spec():
    import importlib.util
    spec_ = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec_)
    spec_.loader.exec_module(mg)
    return mg


def test_oracle_reproduces_reference_fixture(oracle_mod):
    mg = _golden_spec()
    gold = np.load(os.path.join(GOLDEN, "ref_dam16.npz"))
    spec = mg.dam16_spec()
    o = oracle_mod.Oracle(spec.grid_desc(), spec.solver_params(**mg.DAM16_SOLVER), spec.liquid_params(), dbl=False)
    o.set_boundary(spec.boundary)
    pos, vel = scenes.seed(spec, "fp32")
    assert_bitwise(pos, gold["pos0"], "seeded positions")
    o.set_particles(pos, vel)
    for f in ("solidPhi", "liquidWx", "liquidWy", "liquidWz"):
        assert_bitwise(o.field(f), gold[f], f)
    dt = np.float32(spec.dt)
    o.pre_step(dt)
    assert_bitwise(o.field("liquidPhi"), gold["liquidPhi"], "liquidPhi")
    o.particle_to_grid()
    for k in ("vx", "vy", "vz", "wx", "wy", "wz"):
        assert_bitwise(o.field(k), gold["p2g_" + k], "P2G " + k)
    o.apply_gravity(dt)
    assert_bitwise(o.field("vy"), gold["grav_vy"], "gravity")
    st = o.projection(dt)
    assert st["status"] == abi.LHI_OK
    assert_bitwise(o.field("pressure"), gold["pressure"], "pressure")
    assert_bitwise(o.field("rhs"), gold["rhs"], "rhs")
    for lvl in range(4):
        assert_bitwise(o.field("Adiag", lvl), gold[f"Adiag{lvl}"], f"Adiag{lvl}")
        assert_bitwise(o.field("Acoef", lvl), gold[f"Acoef{lvl}"], f"Acoef{lvl}")
    for k in ("vx", "vy", "vz"):
        assert_bitwise(o.field(k), gold["proj_" + k], "projection " + k)
    o.extrapolate(oracle_mod.EXTRAP_SERIAL)
    for k in ("vx", "vy", "vz"):
        assert_bitwise(o.field(k), gold["ext_" + k], "extrapolation " + k)
    assert_bitwise(o.field("isValid"), gold["isValid"], "isValid")
    o.grid_to_particle()
    _, v1, a1 = o.get_particles()
    assert_bitwise(v1, gold["g2p_vel"], "G2P velocity")
    assert_bitwise(a1, gold["g2p_aff"], "G2P affine")
    o.advect_particles(dt)
    assert_bitwise(o.get_particles()[0], gold["pos1"], "advected positions")
    for _ in range(2):
        o.pre_step(dt)
        o.step(dt, oracle_mod.EXTRAP_SERIAL)
    assert_bitwise(o.get_particles()[0], gold["pos3"], "positions after 3 steps")


def test_oracle_matches_reference_build_default_scene(reference_mod):
    """Config/PureLiquid3D.json as the reference ships it (with 16^3 instead
    of 64^3 to keep it quick): Init, then 3 full steps, every stage bitwise."""
    po = reference_mod
    cfg = json.load(open(os.path.join(ROOT, "tests", "golden", "pure_liquid3d.json")))
    cfg["gridDimension"] = [16, 16, 16]
    ref = po.Reference(cfg)
    ref.init()
    sp = cfg["SolverParameter"]
    solver = abi.make_solver_params(sp["maxIterations"], sp["tolerance"], abi.PRECOND_MULTIGRID, sp["numLevel"],
                                    sp["numPreSmooth"], sp["numPostSmooth"], sp["numFinalSmooth"],
                                    sp["smoothingFactor"])
    grid = abi.make_grid_desc(cfg["gridDimension"], cfg["minCoord"], cfg["maxCoord"])
    o = po.Oracle(grid, solver, abi.make_liquid_params(cfg["LiquidParameter"]["density"], cfg["gravity"]))
    o.set_boundary([{"kind": abi.BOUNDARY_NONE, "left": 1},
                    {"kind": abi.BOUNDARY_RECT, "center": (0, 0, 0), "half_extent": (0.9,) * 3, "use_inside": 1}])
    pos, vel, aff = ref.get_particles()
    o.set_particles(pos, vel, aff)
    dt = np.float32(cfg["dt"])
    for step in range(3):
        ref.pre_step(dt)
        o.pre_step(dt)
        assert_bitwise(o.field("liquidPhi"), ref.field("liquidPhi"), f"step {step} liquidPhi")
        ref.step(dt)
        o.step(dt, po.EXTRAP_SERIAL)
        for f in ("vx", "vy", "vz", "pressure", "isValid"):
            assert_bitwise(o.field(f), ref.field(f), f"step {step} {f}")
        for a, b, what in zip(o.get_particles(), ref.get_particles(), ("pos", "vel", "affine")):
            assert_bitwise(a, b, f"step {step} {what}")


def test_reference_pcg_diverges_with_fluid_on_outer_layer(oracle_mod):
    """One-cell walls let fluid cells sit on the domain's outer layer, where
    the reference's PCG updates nothing: its recursion becomes inconsistent
    and diverges.  Updating every fluid cell (REGION_FLUID) restores CG."""
    spec = scenes.dam(16)
    pos, vel = scenes.seed(spec, "fp64")
    res = {}
    for name, solver in (("reference", spec.solver_params(robust=False, tolerance=1e-6,
                                                           tolerance_mode=abi.TOL_RELATIVE)),
                         ("fluid_region", spec.solver_params(robust=False, tolerance=1e-6,
                                                              tolerance_mode=abi.TOL_RELATIVE,
                                                              update_region=abi.REGION_FLUID))):
        o = oracle_mod.Oracle(spec.grid_desc(), solver, spec.liquid_params(), dbl=True)
        o.set_boundary(spec.boundary)
        o.set_particles(pos, vel)
        o.pre_step(spec.dt)
        o.particle_to_grid()
        o.apply_gravity(spec.dt)
        res[name] = o.solve(spec.density, spec.dt)
    assert res["reference"]["status"] != abi.LHI_OK
    assert res["reference"]["true_residual"] > res["reference"]["initial_residual"]
    assert res["fluid_region"]["status"] == abi.LHI_OK


def test_robust_mgpcg_iterations_do_not_grow_with_n(oracle_mod):
    """Reference smoother: iterations ~ N (a diagonal-like preconditioner).
    Damped Gauss-Seidel + flexible CG: about the same count at 16^3 and 32^3."""
    its = {}
    for n in (16, 32):
        spec = scenes.dam(n)
        for robust in (False, True):
            kw = dict(tolerance=1e-6, tolerance_mode=abi.TOL_RELATIVE, update_region=abi.REGION_FLUID,
                      max_iterations=400)
            if robust:
                kw = {}
            o = oracle_mod.Oracle(spec.grid_desc(), spec.solver_params(robust=robust, **kw), spec.liquid_params(),
                                  dbl=True)
            o.set_boundary(spec.boundary)
            o.set_particles(*scenes.seed(spec, "fp64"))
            o.pre_step(spec.dt)
            o.particle_to_grid()
            o.apply_gravity(spec.dt)
            st = o.solve(spec.density, spec.dt)
            assert st["status"] == abi.LHI_OK
            its[(n, robust)] = st["iterations"]
    assert its[(32, False)] > 1.7 * its[(16, False)]
    assert its[(32, True)] <= its[(16, True)] + 3
    assert its[(32, True)] < its[(32, False)] / 3
