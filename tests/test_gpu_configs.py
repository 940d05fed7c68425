"""Parity at the named configurations, against the FP64 oracle.

* dam64 (64^3, seed 0, dt 1/480): FP64 GPU particle positions within
  1e-4 dx of the FP64 oracle after 100 full steps.
* dam128 (64^3's block + the falling sphere, 128^3, seed 1, 5 levels, 2+2
  sweeps): the mixed-precision solve (FP32 V-cycle, FP64 x / dots / true
  residual) stops at ||r||/||b|| <= 1e-6 on the true residual with pressure
  within relative L2 1e-5 of the FP64 oracle solved to 1e-12, on the same
  float inputs; the all-FP64 GPU path is held to the same bar, and to 1e-9
  when both run to 1e-12.
* The PCG body's own SpMV kernel (the TMA-staged tile kernel on the FP32
  grids the fused sweep takes, the row kernel elsewhere) against the oracle's
  GetAx (PressureSolver.cpp:700-717) and its p.Ap sum.
* ComputeDivergence (LiquidModel.cpp:1066-1083): per-cell divergence as the
  reference forms it, the GPU's max-norm bit for bit, its mean against the
  same per-cell values.

The oracle runs its parallel loops on every host core (bit-identical for any
thread count).
"""
import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import assert_close, gpu_model, oracle_model, pair, rel_l2

pytestmark = pytest.mark.gpu

GRID_INPUTS = ("vx", "vy", "vz", "liquidPhi", "liquidWx", "liquidWy", "liquidWz")


def obstacle_scene(n):
    """dam256's boundary (walls + two solid boxes) on an n^3 grid."""
    spec = scenes.dam(n)
    big = scenes.dam256()
    spec.boundary = [dict(big.boundary[0]), scenes.walls(n)] + [dict(b) for b in big.boundary[2:]]
    return spec


@pytest.fixture(scope="module")
def po(oracle_mod):
    oracle_mod.set_threads(0)
    return oracle_mod


def test_c1_dam64_fp64_positions_after_100_steps(po, lhi):
    spec = scenes.dam(64)
    assert spec.seed == 0 and abs(spec.dt - 1.0 / 480.0) < 1e-15
    g, o = pair(po, spec, "fp64")
    its_g, its_o = [], []
    for _ in range(100):
        g.PreStep(spec.dt)
        g.Step(spec.dt)
        o.pre_step(spec.dt)
        st = o.step(spec.dt)
        its_g.append(g.GetSolver().Stats()["iterations"])
        its_o.append(st["iterations"])
        assert st["status"] == abi.LHI_OK
    d = np.abs(g.GetParticleSystem().GetPositions() - o.get_particles()[0]).max()
    assert d <= 1e-4 * spec.dx, (d / spec.dx, its_g, its_o)
    assert max(abs(a - b) for a, b in zip(its_g, its_o)) <= 1


def _solve_on(spec, precision, fields, **solver_over):
    g = gpu_model(spec, precision, spec.solver_params(**solver_over) if solver_over else None)
    for f, v in fields.items():
        g.set_field(f, v)
    st = g.GetSolver().Solve(spec.density, spec.dt)
    p = g.field("pressure")
    g.close()
    return st, p


@pytest.mark.parametrize("steps_before", [0, 40])
def test_c2_dam128_mixed_pressure_vs_fp64_oracle(po, lhi, steps_before):
    spec = scenes.dam128()
    g = gpu_model(spec, "mixed")
    pos, vel = scenes.seed(spec, "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    for _ in range(steps_before):
        g.PreStep(spec.dt)
        g.Step(spec.dt)
    g.PreStep(spec.dt)
    g.Particle2Grid()
    g.ApplyGravity(spec.dt)
    fields = {f: g.field(f) for f in GRID_INPUTS}  # the float inputs every solve below shares
    st_m = g.GetSolver().Solve(spec.density, spec.dt)
    p_mixed = g.field("pressure")
    g.close()
    assert st_m["status"] == abi.LHI_OK, st_m
    assert st_m["true_residual"] <= 1e-6 * st_m["initial_residual"] * 1.0001, st_m

    o = oracle_model(po, spec, "fp64", spec.solver_params(tolerance=1e-12, max_iterations=400))
    for f, v in fields.items():
        o.set_field(f, v.astype(np.float64))
    st_o = o.solve(spec.density, spec.dt)
    assert st_o["status"] == abi.LHI_OK, st_o
    p_o = o.field("pressure")

    f64 = {f: v.astype(np.float64) for f, v in fields.items()}
    st_d, p_d = _solve_on(spec, "fp64", f64)
    st_t, p_t = _solve_on(spec, "fp64", f64, tolerance=1e-12, max_iterations=400)
    assert st_d["status"] == abi.LHI_OK and st_t["status"] == abi.LHI_OK

    err_mixed = rel_l2(p_mixed, p_o)
    err_fp64 = rel_l2(p_d, p_o)
    err_tight = rel_l2(p_t, p_o)
    msg = (f"iterations mixed {st_m['iterations']} fp64 {st_d['iterations']} oracle@1e-12 {st_o['iterations']}; "
           f"rel L2 mixed {err_mixed:.2e} fp64 {err_fp64:.2e} fp64@1e-12 {err_tight:.2e}")
    assert err_mixed <= 1e-5, msg
    assert err_fp64 <= 1e-5, msg
    assert err_tight <= 1e-9, msg
    assert rel_l2(p_mixed, p_d) <= 1e-5, msg


SPMV_CASES = [("dam128", "mixed", True), ("obstacle64", "fp32", True), ("obstacle64", "fp64", False)]


@pytest.mark.parametrize("name,prec,tma", SPMV_CASES)
def test_pcg_spmv_kernel_vs_oracle(po, lhi, name, prec, tma):
    spec = scenes.dam128() if name == "dam128" else obstacle_scene(64)
    g = gpu_model(spec, prec)
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    g.PreStep(spec.dt)
    g.Particle2Grid()
    g.ApplyGravity(spec.dt)
    s = g.GetSolver()
    s.Init()
    s.BuildRHS()
    s.BuildLHS(spec.density, spec.dt)
    o = oracle_model(po, spec, "fp64" if prec == "fp64" else "fp32")
    for f in GRID_INPUTS:
        o.set_field(f, g.field(f))
    o.solver_init()
    o.build_lhs(spec.density, spec.dt)
    wet = g.field("liquidPhi") <= 0
    rng = np.random.default_rng(23)
    p = (rng.standard_normal(wet.size) * wet).astype(g.dtype)
    g.set_field("p", p)
    pap, used_tma = s.SpMV()
    assert used_tma == tma
    ap = g.field("Ap")
    ref = o.get_ax(0, p)
    rtol = 1e-12 if prec == "fp64" else 2e-6
    assert_close(ap[wet], ref[wet], rtol, rtol * np.abs(ref).max(), "A p")
    prod = p[wet].astype(np.float64) * ref[wet].astype(np.float64)
    assert abs(pap - prod.sum()) <= (1e-12 if prec == "fp64" else 1e-5) * np.abs(prod).sum(), (pap, prod.sum())


def _divergence_cells(n, f, dx, dtype):
    """Per-cell divergence of every fluid cell in the reference's order
    (LiquidModel.cpp:1071-1077), in the grid's own float type."""
    vx = f["vx"].reshape(n + 1, n, n)
    vy = f["vy"].reshape(n, n + 1, n)
    vz = f["vz"].reshape(n, n, n + 1)
    lx = f["liquidWx"].reshape(n + 1, n, n)
    ly = f["liquidWy"].reshape(n, n + 1, n)
    lz = f["liquidWz"].reshape(n, n, n + 1)
    d = lx[1:] * vx[1:] - lx[:-1] * vx[:-1]
    d = d + (ly[:, 1:] * vy[:, 1:] - ly[:, :-1] * vy[:, :-1])
    d = d + (lz[:, :, 1:] * vz[:, :, 1:] - lz[:, :, :-1] * vz[:, :, :-1])
    d = (d / dtype(dx)).astype(dtype)
    return d


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("projected", [False, True])
def test_divergence_vs_oracle(po, lhi, prec, projected):
    spec = obstacle_scene(32)
    g, o = pair(po, spec, prec)
    o.pre_step(spec.dt)
    o.particle_to_grid()
    o.apply_gravity(spec.dt)
    if projected:
        o.projection(spec.dt)
    f = {k: o.field(k) for k in GRID_INPUTS}
    for k in ("vx", "vy", "vz", "liquidPhi"):
        g.set_field(k, f[k])
    mean_g, max_g = g.ComputeDivergence(), g.ComputeDivergenceMax()
    mean_o, max_o = o.divergence()
    n = spec.n
    dt = np.float64 if prec == "fp64" else np.float32
    d = _divergence_cells(n, f, o.dx[0], dt)
    wet = f["liquidPhi"].reshape(n, n, n) <= 0
    inner = np.zeros_like(wet)
    inner[1:n - 2, 1:n - 2, 1:n - 2] = True
    exp_max = float(np.abs(d[wet & inner]).max())
    assert max_g == exp_max == max_o, (max_g, exp_max, max_o)
    vals = d[wet].astype(np.float64)
    scale = np.abs(vals).mean()
    assert abs(mean_g - vals.mean()) <= 1e-12 * scale, (mean_g, vals.mean())
    # the oracle sums in the grid's type, as the reference does
    assert abs(mean_o - vals.mean()) <= (1e-12 if prec == "fp64" else 1e-4) * scale, (mean_o, vals.mean())


def test_g2p_factored_mixed_close(po, lhi):
    """Mixed-precision handles gather with the factored (axis-by-axis, fused)
    sums: velocity and affine matrix within rounding of the oracle's
    per-node sums (LiquidModel.cpp:724-823), positions after advection too."""
    spec = obstacle_scene(32)
    g = gpu_model(spec, "mixed")
    o = oracle_model(po, spec, "fp32")
    pos, vel = scenes.seed(spec, "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    o.set_particles(pos, vel)
    rng = np.random.default_rng(17)
    for f in ("vx", "vy", "vz"):
        v = (rng.standard_normal(o.field(f).size) * 2).astype(np.float32)
        o.set_field(f, v)
        g.set_field(f, v)
    o.grid_to_particle()
    g.Grid2Particle()
    _, v_g, a_g = g.GetParticleSystem().GetParticles()
    _, v_o, a_o = o.get_particles()
    assert_close(v_g, v_o, 1e-5, 1e-5 * np.abs(v_o).max(), "velocity")
    assert_close(a_g, a_o, 1e-5, 1e-5 * np.abs(a_o).max(), "affine")
    o.advect_particles(spec.dt)
    g.AdvectParticle(spec.dt)
    d = np.abs(g.GetParticleSystem().GetPositions() - o.get_particles()[0]).max()
    assert d < 1e-5 * spec.dx, d / spec.dx
