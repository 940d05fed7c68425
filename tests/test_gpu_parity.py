"""Per-stage parity of the CUDA path (through the C-ABI) against the CPU
oracle on the same seeded inputs.

Bit-exact where the arithmetic is order-independent or evaluated in the
reference's order: solid SDF and face fractions, the cell sort, the liquid
SDF (cell classification), gravity, RHS and every level's matrix, the
velocity update, extrapolation, G2P and advection.  Tolerance-based where the
sum order differs: P2G (shared-memory accumulation), SpMV (fused
multiply-add), the V-cycle and the pressure solve.
"""
import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import assert_bitwise, assert_close, gpu_model, oracle_model, pair, rel_l2

pytestmark = pytest.mark.gpu

PRECS = ["fp32", "fp64"]


def obstacle_scene(n):
    """dam256's boundary (walls + two solid boxes) on an n^3 grid."""
    spec = scenes.dam(n)
    big = scenes.dam256()
    spec.boundary = [dict(big.boundary[0]), scenes.walls(n)] + [dict(b) for b in big.boundary[2:]]
    return spec


def random_particle_state(po_dtype, n, seed=7):
    rng = np.random.default_rng(seed)
    vel = rng.uniform(-1, 1, size=(n, 3)).astype(po_dtype)
    aff = rng.uniform(-5, 5, size=(n, 9)).astype(po_dtype)
    return vel, aff


@pytest.mark.parametrize("prec", PRECS)
def test_solid_phi_and_face_fractions_bitwise(oracle_mod, lhi, prec):
    spec = obstacle_scene(24)
    g = gpu_model(spec, prec)
    o = oracle_model(oracle_mod, spec, prec)
    for f in ("solidPhi", "liquidWx", "liquidWy", "liquidWz"):
        assert_bitwise(g.field(f), o.field(f), f)


@pytest.mark.parametrize("prec", PRECS)
def test_particle_roundtrip_bitwise(oracle_mod, lhi, prec):
    spec = scenes.dam(16)
    g, o = pair(oracle_mod, spec, prec)
    dt = np.float64 if prec == "fp64" else np.float32
    vel, aff = random_particle_state(dt, o.num_particles())
    pos = o.get_particles()[0]
    g.GetParticleSystem().SetParticles(pos, vel, aff)
    g.sort_particles()  # device order changes, caller order must not
    p2, v2, a2 = g.GetParticleSystem().GetParticles()
    assert_bitwise(p2, pos, "pos")
    assert_bitwise(v2, vel, "vel")
    assert_bitwise(a2, aff, "affine")


@pytest.mark.parametrize("prec", PRECS)
def test_cell_sort_bitwise(oracle_mod, lhi, prec):
    spec = scenes.dam(32)
    g, o = pair(oracle_mod, spec, prec)
    g.sort_particles()
    ids, cs = o.sort_by_cell()
    keys = o.cell_keys()
    assert_bitwise(g.field("particle_id"), ids, "stable order")
    assert_bitwise(g.field("cell_start"), cs, "cell_start")
    assert_bitwise(g.field("cell_key"), keys[ids], "sorted keys")


@pytest.mark.parametrize("prec", PRECS)
def test_cell_sort_after_advection(oracle_mod, lhi, prec):
    """After a step the device order is the previous sort; the new sort must
    still be the stable sort of the caller's order: the oracle's ids, keys
    and cell ranges on the GPU's own positions."""
    spec = scenes.dam(16)
    g, o = pair(oracle_mod, spec, prec)
    for m in (g,):
        m.PreStep(spec.dt)
        m.Step(spec.dt)
    o.pre_step(spec.dt)
    o.step(spec.dt)
    g.sort_particles()
    # oracle keys of the GPU's own positions (G2P/advection are bit-exact)
    o.set_particles(*g.GetParticleSystem().GetParticles())
    keys = o.cell_keys()
    ids = g.field("particle_id")
    assert_bitwise(g.field("cell_key"), keys[ids], "keys")
    cs = g.field("cell_start")
    ids_o, cs_o = o.sort_by_cell()
    assert_bitwise(cs, cs_o, "cell_start")
    assert_bitwise(ids, ids_o, "stable order")


@pytest.mark.parametrize("prec", PRECS)
def test_liquid_phi_bitwise(oracle_mod, lhi, prec):
    spec = scenes.dam(32)
    g, o = pair(oracle_mod, spec, prec)
    g.PreStep(spec.dt)
    o.pre_step(spec.dt)
    assert_bitwise(g.field("liquidPhi"), o.field("liquidPhi"), "liquidPhi")


@pytest.mark.parametrize("prec", PRECS)
def test_p2g_close(oracle_mod, lhi, prec):
    spec = scenes.dam(16)
    g, o = pair(oracle_mod, spec, prec)
    dt = np.float64 if prec == "fp64" else np.float32
    vel, aff = random_particle_state(dt, o.num_particles())
    pos = o.get_particles()[0]
    g.GetParticleSystem().SetParticles(pos, vel, aff)
    o.set_particles(pos, vel, aff)
    g.clear()
    g.Particle2Grid()
    o.clear()
    o.particle_to_grid()
    rtol = 1e-12 if prec == "fp64" else 2e-5
    for f in ("wx", "wy", "wz"):
        a, b = g.field(f), o.field(f)
        assert_close(a, b, rtol, rtol * np.abs(b).max(), f)
    for f in ("vx", "vy", "vz"):
        a, b = g.field(f), o.field(f)
        assert_close(a, b, rtol * 10, rtol * 10 * np.abs(b).max(), f)


def _oracle_after_p2g(oracle_mod, spec, prec, solver=None):
    o = oracle_model(oracle_mod, spec, prec, solver)
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    o.set_particles(pos, vel)
    o.pre_step(spec.dt)
    o.particle_to_grid()
    o.apply_gravity(spec.dt)
    return o


def _copy_grid(o, g, names=("vx", "vy", "vz", "liquidPhi")):
    for f in names:
        g.set_field(f, o.field(f))


@pytest.mark.parametrize("prec", PRECS)
def test_gravity_bitwise(oracle_mod, lhi, prec):
    spec = scenes.dam(16)
    o = oracle_model(oracle_mod, spec, prec)
    g = gpu_model(spec, prec)
    rng = np.random.default_rng(3)
    vy = rng.standard_normal(o.field("vy").size).astype(g.dtype)
    o.set_field("vy", vy)
    g.set_field("vy", vy)
    o.apply_gravity(spec.dt)
    g.ApplyGravity(spec.dt)
    assert_bitwise(g.field("vy"), o.field("vy"), "vy")


@pytest.mark.parametrize("prec", PRECS + ["mixed"])
def test_rhs_and_matrix_bitwise(oracle_mod, lhi, prec):
    spec = obstacle_scene(32)
    solver = spec.solver_params(num_level=4)
    o = _oracle_after_p2g(oracle_mod, spec, prec, solver)
    g = gpu_model(spec, prec, solver)
    _copy_grid(o, g)
    rho, dt = spec.density, spec.dt
    o.solver_init()
    o.build_rhs()
    o.build_lhs(rho, dt)
    s = g.GetSolver()
    s.Init()
    s.BuildRHS()
    s.BuildLHS(rho, dt)
    assert_bitwise(g.field("rhs"), o.field("rhs"), "rhs")
    for lvl in range(4):
        assert_bitwise(g.field("Adiag", lvl), o.field("Adiag", lvl), f"Adiag level {lvl}")
        assert_bitwise(g.field("Acoef", lvl), o.field("Acoef", lvl), f"Acoef level {lvl}")


@pytest.mark.parametrize("prec", PRECS)
def test_spmv_close(oracle_mod, lhi, prec):
    spec = obstacle_scene(32)
    o = _oracle_after_p2g(oracle_mod, spec, prec)
    g = gpu_model(spec, prec)
    _copy_grid(o, g)
    o.solver_init()
    o.build_lhs(spec.density, spec.dt)
    g.GetSolver().Init()
    g.GetSolver().BuildLHS(spec.density, spec.dt)
    rng = np.random.default_rng(5)
    for lvl in range(4):
        n = o.field("Adiag", lvl).size
        x = rng.standard_normal(n).astype(g.dtype)
        a, b = g.GetSolver().GetAx(x, lvl), o.get_ax(lvl, x)
        rtol = 1e-13 if prec == "fp64" else 1e-5
        assert_close(a, b, rtol, rtol * np.abs(b).max(), f"A x level {lvl}")


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("robust", [False, True])
@pytest.mark.parametrize("coarse_cells", [0, 64])
def test_vcycle_close(oracle_mod, lhi, prec, robust, coarse_cells):
    """z after one V-cycle on every cell with phi <= 0.  Air cells are left
    out: their rows are empty, no row reads them, and the active-tile sweeps
    skip the tiles where the dense V-cycle would only prolong values into
    them.  coarse_cells=64 keeps every level above 4^3 on the tile kernels."""
    spec = scenes.dam(32)
    solver = spec.solver_params(robust=robust, coarse_cells=coarse_cells)
    o = _oracle_after_p2g(oracle_mod, spec, prec, solver)
    g = gpu_model(spec, prec, solver)
    _copy_grid(o, g)
    for m in (o,):
        m.solver_init()
        m.build_rhs()
        m.build_lhs(spec.density, spec.dt)
    s = g.GetSolver()
    s.Init()
    s.BuildRHS()
    s.BuildLHS(spec.density, spec.dt)
    r = o.field("rhs") * (o.field("liquidPhi") <= 0)
    o.set_field("r", r)
    g.set_field("r", r)
    o.apply_preconditioner()
    s.ApplyPreconditioner()
    wet = o.field("liquidPhi") <= 0
    err = rel_l2(g.field("z")[wet], o.field("z")[wet])
    assert err < (1e-12 if prec == "fp64" else 1e-4), err


def _solve_pair(oracle_mod, spec, prec, solver, oracle_prec=None):
    o = _oracle_after_p2g(oracle_mod, spec, oracle_prec or prec, solver)
    g = gpu_model(spec, prec, solver)
    _copy_grid(o, g)
    st_g = g.GetSolver().Solve(spec.density, spec.dt)
    st_o = o.solve(spec.density, spec.dt)
    return g, o, st_g, st_o


@pytest.mark.parametrize("prec", PRECS)
def test_solve_reference_flags(oracle_mod, lhi, prec):
    """The reference's own PCG (FR beta, interior region, reference smoother,
    absolute tolerance) on a scene where it is well defined: walls three
    cells thick so no fluid reaches the domain's outer cell layer."""
    spec = scenes.dam(16, wall_cells=3)
    solver = spec.solver_params(robust=False, tolerance=1e-4)
    g, o, st_g, st_o = _solve_pair(oracle_mod, spec, prec, solver)
    assert st_o["status"] == abi.LHI_OK and st_g["status"] == abi.LHI_OK
    assert abs(st_g["iterations"] - st_o["iterations"]) <= (0 if prec == "fp64" else 2)
    err = rel_l2(g.field("pressure"), o.field("pressure"))
    assert err < (1e-9 if prec == "fp64" else 1e-4), err


@pytest.mark.parametrize("prec", PRECS)
def test_solve_robust_flags(oracle_mod, lhi, prec):
    spec = scenes.dam(32)
    # FP32 stores x in float: its true residual stalls near 1e-5 relative, so
    # the FP32 run stops on the recursive residual alone.
    solver = spec.solver_params(true_residual_every=0 if prec == "fp32" else 10)
    g, o, st_g, st_o = _solve_pair(oracle_mod, spec, prec, solver)
    assert st_g["status"] == abi.LHI_OK, st_g
    assert abs(st_g["iterations"] - st_o["iterations"]) <= (0 if prec == "fp64" else 3)
    err = rel_l2(g.field("pressure"), o.field("pressure"))
    assert err < (1e-9 if prec == "fp64" else 1e-3), err


def test_solve_mixed_against_fp64_oracle(oracle_mod, lhi):
    """Mixed precision (FP32 V-cycle, FP64 x and dots, true residual every
    10 iterations) reaches ||r||/||b|| <= 1e-6 on the true residual, and its
    pressure is within relative L2 1e-5 of an FP64 oracle solved to 1e-12."""
    spec = scenes.dam(32)
    g = gpu_model(spec, "mixed")
    o = _oracle_after_p2g(oracle_mod, spec, "fp64", spec.solver_params(tolerance=1e-12, max_iterations=400))
    # identical float inputs for both
    of = _oracle_after_p2g(oracle_mod, spec, "fp32")
    _copy_grid(of, g)
    for f in ("vx", "vy", "vz", "liquidPhi"):
        o.set_field(f, of.field(f).astype(np.float64))
    st_g = g.GetSolver().Solve(spec.density, spec.dt)
    st_o = o.solve(spec.density, spec.dt)
    assert st_g["status"] == abi.LHI_OK
    assert st_g["true_residual"] <= 1e-6 * st_g["initial_residual"] * 1.0001, st_g
    err = rel_l2(g.field("pressure"), o.field("pressure"))
    assert err < 1e-5, err


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_solve_graph_matches_host_loop(oracle_mod, lhi, prec):
    """The device-side loop (CUDA graph with a conditional while node) and
    the host-driven loop run the same kernels in the same order with
    deterministic reductions: identical iterations and bitwise pressure."""
    spec = scenes.dam(32)
    out = []
    for eager in (0, 1):
        solver = spec.solver_params(eager=eager, coarse_cells=64)
        o = _oracle_after_p2g(oracle_mod, spec, prec, solver)
        g = gpu_model(spec, prec, solver)
        _copy_grid(o, g)
        st = g.GetSolver().Solve(spec.density, spec.dt)
        st2 = g.GetSolver().Solve(spec.density, spec.dt)  # graph replay
        assert st["status"] == abi.LHI_OK and st2["iterations"] == st["iterations"]
        out.append((st, g.field("pressure")))
    assert out[0][0]["iterations"] == out[1][0]["iterations"]
    assert_bitwise(out[0][1], out[1][1], "pressure")


@pytest.mark.parametrize("prec", PRECS)
def test_velocity_update_bitwise(oracle_mod, lhi, prec):
    spec = scenes.dam(16)
    o = _oracle_after_p2g(oracle_mod, spec, prec)
    g = gpu_model(spec, prec)
    rng = np.random.default_rng(11)
    p = (rng.standard_normal(o.field("pressure").size) * 100).astype(g.dtype)
    o.set_field("pressure", p)
    _copy_grid(o, g, ("vx", "vy", "vz", "liquidPhi", "pressure"))
    o.velocity_update(spec.dt)
    g.velocity_update(spec.dt)
    for f in ("vx", "vy", "vz"):
        assert_bitwise(g.field(f), o.field(f), f)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("scene", ["dam", "obstacle"])
def test_extrapolate_bitwise(oracle_mod, lhi, prec, scene):
    """Three passes: the first runs the full passes and builds the node
    lists, the later ones walk the lists and see the earlier passes'
    persistent flags."""
    spec = scenes.dam(16) if scene == "dam" else obstacle_scene(16)
    o = _oracle_after_p2g(oracle_mod, spec, prec)
    g, _ = pair(oracle_mod, spec, prec)
    g.clear()
    rng = np.random.default_rng(13)
    for f in ("vx", "vy", "vz"):
        v = rng.standard_normal(o.field(f).size).astype(g.dtype)
        o.set_field(f, v)
        g.set_field(f, v)
    for _ in range(3):
        o.extrapolate(oracle_mod.EXTRAP_JACOBI)
        g.Extrapolate()
        for f in ("vx", "vy", "vz", "tempVx", "tempVy", "tempVz"):
            assert_bitwise(g.field(f), o.field(f), f)
        assert_bitwise(g.field("isValid"), o.field("isValid"), "isValid")


@pytest.mark.parametrize("prec", PRECS)
def test_g2p_and_advect_bitwise(oracle_mod, lhi, prec):
    spec = obstacle_scene(16)
    g, o = pair(oracle_mod, spec, prec)
    rng = np.random.default_rng(17)
    for f in ("vx", "vy", "vz"):
        v = (rng.standard_normal(o.field(f).size) * 2).astype(g.dtype)
        o.set_field(f, v)
        g.set_field(f, v)
    o.grid_to_particle()
    g.Grid2Particle()
    _, v_g, a_g = g.GetParticleSystem().GetParticles()
    _, v_o, a_o = o.get_particles()
    assert_bitwise(v_g, v_o, "velocity")
    assert_bitwise(a_g, a_o, "affine")
    dt = 0.05  # large enough to push particles into the walls and obstacles
    o.advect_particles(dt)
    g.AdvectParticle(dt)
    assert_bitwise(g.GetParticleSystem().GetPositions(), o.get_particles()[0], "positions")


def test_fp64_positions_after_100_steps(oracle_mod, lhi):
    """FP64 GPU path vs FP64 oracle: positions within 1e-4 dx after 100 steps."""
    spec = scenes.dam(16)
    g, o = pair(oracle_mod, spec, "fp64")
    for _ in range(100):
        g.PreStep(spec.dt)
        g.Step(spec.dt)
        o.pre_step(spec.dt)
        o.step(spec.dt)
    d = np.abs(g.GetParticleSystem().GetPositions() - o.get_particles()[0]).max()
    assert d < 1e-4 * spec.dx, d


def test_fp32_steps_track_oracle(oracle_mod, lhi):
    spec = scenes.dam(16)
    g, o = pair(oracle_mod, spec, "fp32")
    for _ in range(10):
        g.PreStep(spec.dt)
        g.Step(spec.dt)
        o.pre_step(spec.dt)
        o.step(spec.dt)
    d = np.abs(g.GetParticleSystem().GetPositions() - o.get_particles()[0]).max()
    assert d < 1e-3 * spec.dx, d


def test_divergence_after_projection(oracle_mod, lhi):
    spec = scenes.dam(32)
    g = gpu_model(spec, "mixed")
    pos, vel = scenes.seed(spec, "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    g.PreStep(spec.dt)
    g.Particle2Grid()
    g.ApplyGravity(spec.dt)
    g.Projection(spec.dt)
    # rhs = -div(u*) per fluid cell; after the update the divergence of the
    # cells whose faces the update touches is the solver's residual
    b = np.abs(g.field("rhs")).max()
    after = g.ComputeDivergenceMax()
    assert b > 0
    assert after < 1e-4 * b, (b, after)
