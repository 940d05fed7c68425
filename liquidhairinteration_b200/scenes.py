"""Seeded dam-break scenes used by the tests and the benchmark.

All inputs are synthetic: a unit-cube MAC grid with one-cell solid walls
(RectBoundary centred at 0.5 with half extent 0.5 - dx, useInside), fluid
primitives seeded with 8 jittered particles per cell by
lhi_scene_seed_particles, zero (or per-primitive) initial velocity, gravity
-9.81 along y and density 1000 as in Config/PureLiquid3D.json.

  dam64   : 64^3,  block [0,0.4]x[0,0.6]x[0,1), seed 0, dt 1/480, 200 steps
  dam128  : 128^3, dam64's block + sphere r=0.15 at (0.7,0.7,0.5) moving
            (0,-1,0), seed 1, 5 MG levels with 2+2 sweeps, 150 steps
  dam256  : 256^3, block [0,0.35]x[0,0.7]x[0,1) + two solid boxes
            [0.55,0.65]x[0,0.3]x[0.2,0.4] and [0.55,0.65]x[0,0.3]x[0.6,0.8],
            seed 3, dt 1/960, 100 steps, 6 MG levels with 2+2 sweeps (w 1.1)
  damN    : any N with dam64's layout (small parity cases)
  batch   : random_scene(): the batched form's scenes -- grid size from
            {32, 48, 64, 96}, 1-4 fluid primitives (axis boxes with sides
            U[0.15, 0.5], spheres with radius U[0.1, 0.25], centres inside
            the walls), 0-3 solid boxes covering 5-15% of the volume
"""
from dataclasses import dataclass, field

import numpy as np

from . import abi

# Solver flags.  REFERENCE reproduces CGSolver<3>::Solve as written (absolute
# tolerance from the JSON).  ROBUST is the consistent solver the dam-break
# scenes need: the reference's update region and smoother make its PCG
# diverge once fluid reaches the domain's outer cell layer, and its smoother
# (z_GS / 2 for w = 0.5) turns the V-cycle into a diagonal-like
# preconditioner; ROBUST updates every fluid cell, smooths with plain damped
# Gauss-Seidel (w = 1) and uses flexible (Polak-Ribiere) CG with a true
# residual every 10 iterations.
REFERENCE_SOLVER = dict(tolerance_mode=abi.TOL_ABSOLUTE, cg_variant=abi.CG_REFERENCE,
                        update_region=abi.REGION_INTERIOR, smoother=abi.SMOOTHER_REFERENCE,
                        smoothing_factor=0.5, true_residual_every=0)
ROBUST_SOLVER = dict(tolerance=1e-6, tolerance_mode=abi.TOL_RELATIVE, cg_variant=abi.CG_FLEXIBLE,
                     update_region=abi.REGION_FLUID, smoother=abi.SMOOTHER_DAMPED_GS, smoothing_factor=1.0,
                     true_residual_every=10, max_iterations=200)


@dataclass
class SceneSpec:
    name: str
    n: int
    boundary: list
    prims: list
    seed: int
    dt: float
    steps: int
    solver: dict = field(default_factory=dict)
    robust_solver: dict = field(default_factory=dict)  # the scene's tuning of the ROBUST flags
    density: float = 1000.0
    gravity: float = -9.81

    @property
    def dx(self):
        return 1.0 / self.n

    def grid_desc(self):
        return abi.make_grid_desc((self.n,) * 3, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))

    def solver_params(self, robust=True, **over):
        """JSON solver parameters (4 levels, 5/5/20 sweeps, w 0.5, 100
        iterations) with the scene's overrides, then ROBUST_SOLVER (default,
        with the scene's tuning of it) or REFERENCE_SOLVER flags, then
        ``over``."""
        s = dict(max_iterations=100, tolerance=1e-5, preconditioner=abi.PRECOND_MULTIGRID, num_level=4,
                 num_pre_smooth=5, num_post_smooth=5, num_final_smooth=20, smoothing_factor=0.5)
        s.update(self.solver)
        s.update(ROBUST_SOLVER if robust else REFERENCE_SOLVER)
        if robust:
            s.update(self.robust_solver)
        s.update(over)
        return abi.make_solver_params(**s)

    def liquid_params(self, **over):
        p = dict(density=self.density, gravity=self.gravity)
        p.update(over)
        return abi.make_liquid_params(**p)

    def config_json(self, solver=None):
        """The scene in the reference's JSON schema (Config/PureLiquid3D.json)."""
        sp = solver or self.solver_params()
        pre = {abi.PRECOND_NONE: "None", abi.PRECOND_JACOBI: "Jacobi",
               abi.PRECOND_MULTIGRID: "Multigrid"}[sp.preconditioner]
        return {
            "SolverParameter": {"maxIterations": sp.max_iterations, "tolerance": sp.tolerance,
                                "preconditionerType": pre, "numLevel": sp.num_level,
                                "numPreSmooth": sp.num_pre_smooth, "numPostSmooth": sp.num_post_smooth,
                                "numFinalSmooth": sp.num_final_smooth,
                                "smoothingFactor": sp.smoothing_factor},
            "LiquidParameter": {"numParticles": 0, "viscosity": 0.001, "density": self.density,
                                "surfaceTension": 0.0728, "correctCycle": 8},
            "HairParameter": {"radius": 0.05, "youngsModulus": 1e5, "shearModulus": 1e5, "viscosity": 1000.0,
                              "density": 1000.0, "refRotation": 0.0, "accumViscosity": True, "numHair": 0,
                              "numParticles": 0, "info": []},
            "dt": self.dt, "gravity": self.gravity, "gridDimension": [self.n] * 3,
            "minCoord": [0.0, 0.0, 0.0], "maxCoord": [1.0, 1.0, 1.0],
        }


def walls(n, cells=1):
    """Unit-cube walls ``cells`` cells thick: solid outside [c dx, 1 - c dx]^3.
    With cells >= 3 no particle's SDF window reaches the outer cell layer, so
    the reference's own solver stays well defined there."""
    dx = 1.0 / n
    return {"kind": abi.BOUNDARY_RECT, "center": (0.5, 0.5, 0.5), "half_extent": (0.5 - cells * dx,) * 3,
            "use_inside": 1}


def box(lo, hi, solid=True):
    c = tuple((a + b) / 2 for a, b in zip(lo, hi))
    h = tuple((b - a) / 2 for a, b in zip(lo, hi))
    return {"kind": abi.BOUNDARY_RECT, "center": c, "half_extent": h, "use_inside": 0 if solid else 1}


def dam(n, seed=0, steps=200, dt=1.0 / 480.0, wall_cells=1):
    return SceneSpec(
        name=f"dam{n}", n=n,
        boundary=[{"kind": abi.BOUNDARY_NONE, "left": 1}, walls(n, wall_cells)],
        prims=[{"kind": abi.FLUID_BOX, "a": (0.0, 0.0, 0.0), "b": (0.4, 0.6, 1.0)}],
        seed=seed, dt=dt, steps=steps)


def dam128():
    s = dam(128, seed=1, steps=150)
    s.name = "dam128"
    s.prims = s.prims + [{"kind": abi.FLUID_SPHERE, "a": (0.7, 0.7, 0.5), "b": (0.15, 0.0, 0.0),
                          "velocity": (0.0, -1.0, 0.0)}]
    s.solver = dict(num_level=5, num_pre_smooth=2, num_post_smooth=2)
    return s


def dam256():
    n = 256
    return SceneSpec(
        name="dam256", n=n,
        boundary=[{"kind": abi.BOUNDARY_UNION, "left": 1, "right": 2}, walls(n),
                  {"kind": abi.BOUNDARY_UNION, "left": 3, "right": 4},
                  box((0.55, 0.0, 0.2), (0.65, 0.3, 0.4)), box((0.55, 0.0, 0.6), (0.65, 0.3, 0.8))],
        prims=[{"kind": abi.FLUID_BOX, "a": (0.0, 0.0, 0.0), "b": (0.35, 0.7, 1.0)}],
        seed=3, dt=1.0 / 960.0, steps=100,
        # 6 levels (256^3 down to 8^3): 15-16 PCG iterations per solve against
        # 21 with 5 levels, 7 levels needs 22 (the 4^3 level's coarse correction
        # is too rough); 2+2 sweeps beat 3+3 and 1+1 on time to solution; the
        # sweeps over-relaxed by 1.1 take 13-15 (1.0: 15-16, 1.2: 16, 0.9: 19)
        solver=dict(num_level=6, num_pre_smooth=2, num_post_smooth=2),
        robust_solver=dict(smoothing_factor=1.1))


def random_scene(rng, n=None, sizes=(32, 48, 64, 96), steps=100, dt=1.0 / 480.0, seed=None):
    """One scene of the batched form, drawn from ``rng`` (numpy Generator)."""
    n = int(n if n is not None else rng.choice(sizes))
    lo, hi = 1.5 / n, 1.0 - 1.5 / n
    prims = []
    for _ in range(int(rng.integers(1, 5))):
        if rng.uniform() < 0.5:
            side = rng.uniform(0.15, 0.5, size=3)
            c = rng.uniform(lo + side / 2, hi - side / 2)
            prims.append({"kind": abi.FLUID_BOX, "a": tuple(c - side / 2), "b": tuple(c + side / 2)})
        else:
            rad = rng.uniform(0.1, 0.25)
            c = rng.uniform(lo + rad, hi - rad, size=3)
            prims.append({"kind": abi.FLUID_SPHERE, "a": tuple(c), "b": (rad, 0.0, 0.0)})
    nsolid = int(rng.integers(0, 4))
    boxes = []
    if nsolid:
        frac = rng.uniform(0.05, 0.15) / nsolid
        for _ in range(nsolid):
            aspect = rng.uniform(0.5, 2.0, size=3)
            side = np.clip(aspect * frac ** (1.0 / 3.0) / np.prod(aspect) ** (1.0 / 3.0), 0.05, 0.8)
            c = rng.uniform(lo + side / 2, hi - side / 2)
            boxes.append(box(tuple(c - side / 2), tuple(c + side / 2)))
    # union tree: node 0 = walls U solids
    boundary = [{"kind": abi.BOUNDARY_NONE, "left": 1}, walls(n)]
    for b in boxes:
        root = dict(boundary[0])
        boundary[0] = {"kind": abi.BOUNDARY_UNION, "left": len(boundary), "right": len(boundary) + 1}
        boundary.append(root if root["kind"] != abi.BOUNDARY_NONE else walls(n))
        boundary.append(b)
    return SceneSpec(name=f"batch{n}", n=n, boundary=boundary, prims=prims,
                     seed=int(seed if seed is not None else rng.integers(0, 2 ** 31)), dt=dt, steps=steps,
                     solver=dict(num_level=4 if n <= 64 else 5, num_pre_smooth=2, num_post_smooth=2))


def get(name):
    if name == "dam64":
        return dam(64)
    if name == "dam128":
        return dam128()
    if name == "dam256":
        return dam256()
    if name.startswith("dam"):
        return dam(int(name[3:]))
    raise KeyError(name)


def seed(spec, precision="fp32"):
    """(positions, velocities) of the scene's seeded particles."""
    from .model import seed_particles
    return seed_particles(spec.grid_desc(), spec.boundary, spec.prims, spec.seed, precision)


def build(spec, precision="fp32", solver=None, **liquid_over):
    """A LiquidModel on the GPU with the scene's boundary and particles."""
    from .model import LiquidModel
    m = LiquidModel.from_params(spec.grid_desc(), solver or spec.solver_params(),
                                spec.liquid_params(**liquid_over), precision)
    arr = abi.boundary_array(spec.boundary)
    from ._lib import call
    call("lhi_liquid_set_boundary", m._h, arr, len(spec.boundary), 0)
    pos, vel = seed(spec, precision)
    m.GetParticleSystem().SetParticles(pos, vel)
    return m


def particle_count(spec):
    from .model import seed_particles  # noqa: F401
    import ctypes as C
    from ._lib import call
    n = C.c_int64()
    call("lhi_scene_seed_particles", C.byref(spec.grid_desc()), abi.boundary_array(spec.boundary),
         len(spec.boundary), 0, abi.fluid_array(spec.prims), len(spec.prims), int(spec.seed),
         abi.PRECISION_FP32, C.byref(n), None, None)
    return n.value


def as_numpy_dtype(precision):
    return np.float64 if precision == "fp64" else np.float32
