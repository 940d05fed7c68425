"""Python host mirror of the reference's liquid call surface.

``Scene`` / ``LiquidModel`` / ``CGSolver`` / ``ParticleSystem`` and the
boundary classes keep the reference's names, argument meaning and error
behaviour (a failing call raises, like the reference's exceptions); every
operation runs on the GPU through liblhi.so.

Reference surfaces mirrored:
  Scene<3>            Scene.h:13-48, Scene.cpp:13-20
  LiquidModel<3>      LiquidModel.h:14-61
  CGSolver<3>         PressureSolver.h:81-118
  ParticleSystem<3>   ParticleSystem.h:24-60
  BaseBoundary<3>...  Boundary.h:6-96
  Solver/Liquid/SceneParameter  SceneParameter.h:10-153
"""
import ctypes as C
import json

import numpy as np

from . import abi
from ._lib import call, lib

PRECISIONS = {"fp32": abi.PRECISION_FP32, "mixed": abi.PRECISION_MIXED, "fp64": abi.PRECISION_FP64}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ------------------------------------------------------------- parameters
class SolverParameter:
    """SolverParameter<3> (SceneParameter.h:10-45) plus the new solver keys:
    toleranceMode ("absolute" | "relative"), cgVariant ("reference" |
    "flexible") and trueResidualEvery (int)."""

    _PRE = {"None": abi.PRECOND_NONE, "Jacobi": abi.PRECOND_JACOBI, "Multigrid": abi.PRECOND_MULTIGRID,
            "Learned": abi.PRECOND_LEARNED}

    def __init__(self, cfg):
        s = cfg["SolverParameter"]
        self.maxIterations = int(s["maxIterations"])
        self.tolerance = float(s["tolerance"])
        self.numLevel = int(s["numLevel"])
        self.numPreSmooth = int(s["numPreSmooth"])
        self.numPostSmooth = int(s["numPostSmooth"])
        self.numFinalSmooth = int(s["numFinalSmooth"])
        self.smoothingFactor = float(s["smoothingFactor"])
        t = s["preconditionerType"]
        if t not in self._PRE:
            raise RuntimeError("Unknown preconditioner type")
        self.preconditionerType = t
        self.toleranceMode = s.get("toleranceMode", "absolute")
        self.cgVariant = s.get("cgVariant", "reference")
        self.trueResidualEvery = int(s.get("trueResidualEvery", 0))

    def to_abi(self):
        return abi.make_solver_params(
            self.maxIterations, self.tolerance, self._PRE[self.preconditionerType], self.numLevel,
            self.numPreSmooth, self.numPostSmooth, self.numFinalSmooth, self.smoothingFactor,
            abi.TOL_RELATIVE if self.toleranceMode == "relative" else abi.TOL_ABSOLUTE,
            abi.CG_FLEXIBLE if self.cgVariant == "flexible" else abi.CG_REFERENCE, self.trueResidualEvery)


class LiquidParameter:
    """LiquidParameter<3> (SceneParameter.h:48-66)."""

    def __init__(self, cfg):
        s = cfg["LiquidParameter"]
        self.density = float(s["density"])
        self.viscosity = float(s["viscosity"])
        self.numParticles = int(s["numParticles"])
        self.surfaceTension = float(s["surfaceTension"])
        self.correctCycle = int(s["correctCycle"])


class SceneParameter:
    """SceneParameter<3> (SceneParameter.h:132-152)."""

    def __init__(self, cfg):
        self.dt = float(cfg["dt"])
        self.gravity = float(cfg["gravity"])
        self.minCoord = tuple(float(v) for v in cfg["minCoord"][:3])
        self.maxCoord = tuple(float(v) for v in cfg["maxCoord"][:3])
        self.gridDimension = tuple(int(v) for v in cfg["gridDimension"][:3])


# ------------------------------------------------------------- boundaries
class BaseBoundary:
    """BaseBoundary<3> (Boundary.h:6-27): an SDF tree node, negative = solid."""

    def __init__(self):
        self.left = None
        self.right = None

    def SetChild(self, b):
        self.left = b

    def SetLeftChild(self, b):
        self.left = b

    def SetRightChild(self, b):
        self.right = b

    def nodes(self):
        """Flattened tree for the C-ABI; index 0 is this node."""
        out = []

        def rec(b):
            i = len(out)
            out.append(None)
            d = b._node()
            if b.left is not None:
                d["left"] = rec(b.left)
            if b.right is not None:
                d["right"] = rec(b.right)
            out[i] = d
            return i

        rec(self)
        return out

    def Compute(self, pos, precision="fp32"):
        """Evaluate the SDF at points (n x 3) on the host."""
        prec = PRECISIONS[precision]
        dt = np.float64 if prec == abi.PRECISION_FP64 else np.float32
        pts = np.ascontiguousarray(pos, dtype=dt).reshape(-1, 3)
        out = np.empty(pts.shape[0], dt)
        nodes = self.nodes()
        arr = abi.boundary_array(nodes)
        call("lhi_boundary_eval", arr, len(nodes), 0, prec, _ptr(pts), pts.shape[0], _ptr(out))
        return out


class OperatorBoundary(BaseBoundary):
    """OperatorBoundary<3> (Boundary.h:29-62)."""

    Union, Intersection, Substract, NoneType = "Union", "Intersection", "Substract", "None"
    _K = {"Union": abi.BOUNDARY_UNION, "Intersection": abi.BOUNDARY_INTERSECTION,
          "Substract": abi.BOUNDARY_SUBTRACT, "None": abi.BOUNDARY_NONE}

    def __init__(self, op="None", left=None, right=None):
        super().__init__()
        if op not in self._K:
            raise RuntimeError("Failed to recognize OperatorType")
        self.op = op
        self.left, self.right = left, right

    def _node(self):
        return {"kind": self._K[self.op]}


class SolidBoundary(BaseBoundary):
    """SolidBoundary<3> (Boundary.h:64-77): Compute() returns 1."""

    def __init__(self, center=(0, 0, 0), useInside=False):
        super().__init__()
        self.center = tuple(center)
        self.useInside = bool(useInside)

    def _node(self):
        return {"kind": abi.BOUNDARY_SOLID, "center": self.center, "use_inside": int(self.useInside)}


class RectBoundary(SolidBoundary):
    """RectBoundary<3> (Boundary.h:79-95): box SDF, sign flipped by useInside."""

    def __init__(self, center, halfExtent, useInside=False):
        super().__init__(center, useInside)
        self.halfExtent = tuple(halfExtent)

    def _node(self):
        return {"kind": abi.BOUNDARY_RECT, "center": self.center, "half_extent": self.halfExtent,
                "use_inside": int(self.useInside)}


# ------------------------------------------------------------------- model
class ParticleSystem:
    """ParticleSystem<3> view on the device state (ParticleSystem.h:24-60).
    Getters download in the caller's particle order; setters upload."""

    def __init__(self, model):
        self._m = model

    def NumParticles(self):
        n = C.c_int64()
        call("lhi_liquid_num_particles", self._m._h, C.byref(n))
        return n.value

    def GetParticles(self):
        """(positions n x 3, velocities n x 3, affine n x 9 column-major)."""
        n = self.NumParticles()
        dt = self._m.dtype
        pos, vel, aff = np.empty((n, 3), dt), np.empty((n, 3), dt), np.empty((n, 9), dt)
        if n:
            call("lhi_liquid_get_particles", self._m._h, _ptr(pos), _ptr(vel), _ptr(aff))
        return pos, vel, aff

    def GetPositions(self):
        return self.GetParticles()[0]

    def SetParticles(self, pos, vel=None, affine=None):
        dt = self._m.dtype
        pos = np.ascontiguousarray(pos, dtype=dt).reshape(-1, 3)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=dt).reshape(-1, 3)
        affine = None if affine is None else np.ascontiguousarray(affine, dtype=dt).reshape(-1, 9)
        call("lhi_liquid_set_particles", self._m._h, pos.shape[0], _ptr(pos), _ptr(vel), _ptr(affine))

    def GetRadius(self, index=0):
        return self._m.radius

    def SpawnParticles(self, minCoord, maxCoord, maxCount=None):
        """ParticleSystem<3>::SpawnParticles (ParticleSystem.cpp:45-64)."""
        pos = spawn_lattice(minCoord, maxCoord, self._m.radius, maxCount if maxCount is not None else 2 ** 62,
                            self._m.precision)
        self.SetParticles(pos)
        return pos.shape[0]

    def WriteToFile(self, filename, isAppend=False):
        """ParticleSystem::WriteToFile (ParticleSystem.cpp:67-85): count line
        then comma-separated positions, std::ostream default formatting."""
        from . import snapshots
        snapshots.write_frame(filename, self.GetPositions(), append=isAppend)

    def _meta(self):
        g = self._m.grid
        return {"precision": self._m.precision, "grid_dim": list(g.dim),
                "min_coord": list(g.min_coord), "max_coord": list(g.max_coord)}

    def SaveCheckpoint(self, filename, **counters):
        """Binary checkpoint of the whole particle state (exact bits), the
        model's precision and grid, and the caller's counters (e.g. step and
        time).  Stepping a model loaded from it under the same solver and
        liquid parameters tracks the uninterrupted run to rounding: the cell
        order is the same (ties go by particle id), but P2G's atomic adds
        land in a run-dependent order."""
        from . import snapshots
        pos, vel, aff = self.GetParticles()
        snapshots.save_checkpoint(filename, pos, vel, aff, meta=self._meta(), **counters)

    def LoadCheckpoint(self, filename):
        """Restores a SaveCheckpoint file; returns its counters.  A file
        saved with another precision or grid raises ValueError and leaves
        the particles as they were."""
        from . import snapshots
        c = snapshots.load_checkpoint(filename, meta=self._meta())
        self.SetParticles(c.pop("pos"), c.pop("vel"), c.pop("affine"))
        return c


class CGSolver:
    """CGSolver<3> (PressureSolver.h:81-118) bound to a LiquidModel's grid."""

    def __init__(self, model):
        self._m = model

    def Init(self):
        call("lhi_solver_init", self._m._h)

    def BuildRHS(self):
        call("lhi_solver_build_rhs", self._m._h)

    def BuildLHS(self, liquidDensity, dt):
        call("lhi_solver_build_lhs", self._m._h, float(liquidDensity), float(dt))

    def ApplyPreconditioner(self):
        call("lhi_solver_apply_preconditioner", self._m._h)

    def Solve(self, liquidDensity, dt, check=False):
        """Returns the solve statistics dict; check=True raises when the
        solve stops at the iteration cap."""
        st = abi.SolveStats()
        rc = lib().lhi_solver_solve(self._m._h, float(liquidDensity), float(dt), C.byref(st))
        if rc not in (abi.LHI_OK, abi.LHI_E_NOT_CONVERGED) or (check and rc != abi.LHI_OK):
            from ._lib import check as _check
            _check(rc, "lhi_solver_solve")
        return st.as_dict()

    def GetAx(self, x, level=0):
        x = np.ascontiguousarray(x, dtype=self._m.dtype)
        out = np.empty_like(x)
        call("lhi_solver_get_ax", self._m._h, int(level), _ptr(x), _ptr(out))
        return out

    def SpMV(self):
        """One SpMV of the PCG body on the solver's p (field "p") with the
        solve's own kernel; writes field "Ap" and returns (p.Ap over the
        update region, True when the TMA-staged tile kernel ran)."""
        d, t = C.c_double(), C.c_int32()
        call("lhi_solver_spmv", self._m._h, C.byref(d), C.byref(t))
        return d.value, bool(t.value)

    def SetNetwork(self, net, fallbackIterations=0):
        """The learned preconditioner's network (handle created with
        preconditionerType "Learned"); the handle keeps a reference."""
        call("lhi_solver_set_network", self._m._h, net._h, int(fallbackIterations))
        self._net = net

    def LearnedStats(self):
        """(iterations that used the network, iteration where the V-cycle
        fallback started or -1) of the last solve."""
        a, b = C.c_int32(), C.c_int32()
        call("lhi_solver_learned_stats", self._m._h, C.byref(a), C.byref(b))
        return a.value, b.value

    def RecordResiduals(self, maxSnapshots):
        call("lhi_solver_record_residuals", self._m._h, int(maxSnapshots))

    def NumSnapshots(self):
        n = C.c_int32()
        call("lhi_solver_num_snapshots", self._m._h, C.byref(n))
        return n.value

    def ActiveTiles(self, level=0):
        """(active tiles, total tiles, solved by the coarse CTA) of a level."""
        a, t, c = C.c_int32(), C.c_int32(), C.c_int32()
        call("lhi_solver_active_tiles", self._m._h, int(level), C.byref(a), C.byref(t), C.byref(c))
        return a.value, t.value, bool(c.value)

    def Stats(self):
        st = abi.SolveStats()
        call("lhi_solver_get_stats", self._m._h, C.byref(st))
        return st.as_dict()


class LiquidModel:
    """LiquidModel<3> (LiquidModel.h:14-82) on one B200.

    ``LiquidModel(scene)`` like the reference, or ``LiquidModel.from_params``.
    """

    def __init__(self, scene, precision="fp32", particle_radius=0.0):
        self._h = None
        self.scene = scene
        self._create(scene.grid_desc(), scene.solver.to_abi(),
                     abi.make_liquid_params(scene.liquid.density, scene.params.gravity, particle_radius),
                     precision)

    @classmethod
    def from_params(cls, grid, solver, liquid, precision="fp32"):
        self = cls.__new__(cls)
        self._h = None
        self.scene = None
        self._create(grid, solver, liquid, precision)
        return self

    def _create(self, grid, solver, liquid, precision):
        self.precision = precision
        prec = PRECISIONS[precision]
        self.dtype = np.float64 if prec == abi.PRECISION_FP64 else np.float32
        h = C.c_void_p()
        call("lhi_liquid_create", C.byref(grid), C.byref(solver), C.byref(liquid), prec, C.byref(h))
        self._h = h
        self.grid = grid
        self.solver_params = solver
        self.liquid_params = liquid
        self.dim = tuple(grid.dim)
        d = (C.c_double * 3)()
        call("lhi_liquid_get_dx", self._h, d)
        self.dx = tuple(d)
        self.radius = liquid.particle_radius if liquid.particle_radius > 0 else float(self.dtype(2) * self.dtype(self.dx[0]))
        self.m_boundary = None
        self.m_ps = ParticleSystem(self)
        self.m_solver = CGSolver(self)

    def close(self):
        if self._h:
            lib().lhi_liquid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference surface
    def Init(self):
        """LiquidModel<3>::Init (LiquidModel.cpp:507-512)."""
        self.ComputeSolidPhi()
        mn = np.array([self.grid.min_coord[i] for i in range(3)], self.dtype)
        mx = np.array([self.grid.max_coord[i] for i in range(3)], self.dtype)
        off = self.dtype(0.3) * (mx - mn)
        n = self.scene.liquid.numParticles if self.scene is not None else 2 ** 62
        self.m_ps.SpawnParticles((mn + off).astype(np.float64), (mx - off).astype(np.float64), n)

    def PreStep(self, dt):
        call("lhi_liquid_pre_step", self._h, float(dt))

    def Step(self, dt):
        call("lhi_liquid_step", self._h, float(dt))

    def PostStep(self, dt):
        call("lhi_liquid_post_step", self._h, float(dt))

    def ComputeLiquidPhi(self):
        call("lhi_liquid_compute_liquid_phi", self._h)

    def ComputeSolidPhi(self):
        if self.m_boundary is None:
            return
        nodes = self.m_boundary.nodes()
        call("lhi_liquid_set_boundary", self._h, abi.boundary_array(nodes), len(nodes), 0)

    def Particle2Grid(self):
        call("lhi_liquid_particle_to_grid", self._h)

    def Grid2Particle(self):
        call("lhi_liquid_grid_to_particle", self._h)

    def Projection(self, dt):
        call("lhi_liquid_projection", self._h, float(dt))

    SolvePressure = Projection

    def ApplyGravity(self, dt):
        call("lhi_liquid_apply_gravity", self._h, float(dt))

    def AdvectParticle(self, dt):
        call("lhi_liquid_advect_particles", self._h, float(dt))

    def Extrapolate(self):
        call("lhi_liquid_extrapolate", self._h)

    def CorrectVolume(self, dt):
        """LiquidModel<3>::CorrectVolume (LiquidModel.cpp:1086-1132) on the GPU
        (lhi_liquid_correct_volume).  The reference's Step has the call
        commented out (LiquidModel.cpp:527); Step makes it only when the
        handle was created with correct_volume set."""
        call("lhi_liquid_correct_volume", self._h, float(dt))

    def ComputeDivergence(self):
        m, mx = C.c_double(), C.c_double()
        call("lhi_liquid_compute_divergence", self._h, C.byref(m), C.byref(mx))
        return m.value

    def ComputeDivergenceMax(self):
        m, mx = C.c_double(), C.c_double()
        call("lhi_liquid_compute_divergence", self._h, C.byref(m), C.byref(mx))
        return mx.value

    def GetCFL(self):
        d = C.c_double()
        call("lhi_liquid_get_cfl", self._h, C.byref(d))
        return d.value

    def Render(self, width=480, height=480, pointSize=5.0, color=(0, 0, 255, 255),
               background=(255, 255, 255, 255), ndc=False):
        """LiquidModel<3>::Render without a display (lhi_liquid_render): the
        particles drawn as the reference's shaders draw them into an RGBA
        image (height x width x 4, row 0 at the bottom as in GL).  With
        ndc=True also returns the vertex shader's coordinates (n x 3)."""
        rp = abi.make_render_params(width, height, pointSize, color, background)
        img = np.empty((height, width, 4), np.uint8)
        out = np.empty((self.GetParticleSystem().NumParticles(), 3), np.float32) if ndc else None
        call("lhi_liquid_render", self._h, C.byref(rp), _ptr(out), _ptr(img))
        return (img, out) if ndc else img

    def SetBoundary(self, boundary):
        self.m_boundary = boundary

    def GetParticleSystem(self):
        return self.m_ps

    def GetSolver(self):
        return self.m_solver


    # -- extras
    def sort_particles(self):
        call("lhi_liquid_sort_particles", self._h)

    def clear(self):
        call("lhi_liquid_clear", self._h)

    def velocity_update(self, dt):
        call("lhi_liquid_velocity_update", self._h, float(dt))

    def sync(self):
        call("lhi_liquid_sync", self._h)

    def stream_ptr(self):
        """cudaStream_t of the handle (all its device work runs on it)."""
        s = C.c_void_p()
        call("lhi_liquid_stream", self._h, C.byref(s))
        return s.value or 0

    def profile(self, enable=True):
        call("lhi_liquid_profile", self._h, 1 if enable else 0)

    def profile_read(self):
        """{category: (timed launches, total device ms)} since profile(True)."""
        out = {}
        for i, name in enumerate(abi.KERNEL_CATEGORIES):
            n, ms = C.c_int64(), C.c_double()
            call("lhi_liquid_profile_read", self._h, i, C.byref(n), C.byref(ms))
            out[name] = (n.value, ms.value)
        return out

    def set_solid_phi(self, node_phi):
        a = np.ascontiguousarray(node_phi, dtype=self.dtype)
        call("lhi_liquid_set_solid_phi", self._h, _ptr(a))

    def field(self, name, level=0):
        f = abi.FIELD_NAMES[name] if isinstance(name, str) else int(name)
        cnt, eb = C.c_int64(), C.c_int32()
        call("lhi_liquid_field_size", self._h, f, int(level), C.byref(cnt), C.byref(eb))
        ints = (abi.FIELD_CELL_KEY, abi.FIELD_PARTICLE_ID, abi.FIELD_CELL_START)
        dt = {1: np.uint8, 4: (np.int32 if f in ints else np.float32), 8: np.float64}[eb.value]
        out = np.empty(cnt.value, dt)
        if cnt.value:
            call("lhi_liquid_get_field", self._h, f, int(level), _ptr(out))
        return out

    def set_field(self, name, data, level=0):
        f = abi.FIELD_NAMES[name] if isinstance(name, str) else int(name)
        cnt, eb = C.c_int64(), C.c_int32()
        call("lhi_liquid_field_size", self._h, f, int(level), C.byref(cnt), C.byref(eb))
        dt = {1: np.uint8, 4: np.float32, 8: np.float64}[eb.value]
        a = np.ascontiguousarray(data, dtype=dt).reshape(-1)
        if a.size != cnt.value:
            raise ValueError(f"field {name}: expected {cnt.value} values, got {a.size}")
        call("lhi_liquid_set_field", self._h, f, int(level), _ptr(a))


class Scene:
    """Scene<3> (Scene.h:13-48, Scene.cpp:13-20): parses the reference's JSON
    config (file path or dict), builds the LiquidModel and the default box
    boundary RectBoundary(0, 0.9, useInside)."""

    def __init__(self, config, precision="fp32"):
        cfg = json.load(open(config)) if isinstance(config, str) else dict(config)
        self.config = cfg
        self.solver = SolverParameter(cfg)
        self.liquid = LiquidParameter(cfg)
        self.params = SceneParameter(cfg)
        self.m_boundary = OperatorBoundary("None")
        self.m_boundary.SetChild(RectBoundary((0, 0, 0), (0.9, 0.9, 0.9), True))
        self.m_liquidModel = LiquidModel(self, precision)
        self.m_liquidModel.SetBoundary(self.m_boundary)

    def grid_desc(self):
        return abi.make_grid_desc(self.params.gridDimension, self.params.minCoord, self.params.maxCoord)

    def GetLiquidModel(self):
        return self.m_liquidModel

    def GetSolverParameter(self):
        return self.solver

    def GetLiquidParameter(self):
        return self.liquid

    def GetSceneParameter(self):
        return self.params

    def GetLiquidDensity(self):
        return self.liquid.density

    def GetGravity(self):
        return self.params.gravity

    def GetMinCoord(self):
        return self.params.minCoord

    def GetMaxCoord(self):
        return self.params.maxCoord

    def GetGridDimension(self):
        return self.params.gridDimension


def kernel_launch_count():
    n = C.c_int64()
    call("lhi_kernel_launch_count", C.byref(n))
    return n.value


# --------------------------------------------------------- scene builders
def spawn_lattice(min_coord, max_coord, default_radius, max_count, precision="fp32"):
    prec = PRECISIONS[precision]
    dt = np.float64 if prec == abi.PRECISION_FP64 else np.float32
    mn = (C.c_double * 3)(*min_coord)
    mx = (C.c_double * 3)(*max_coord)
    n = C.c_int64()
    call("lhi_scene_spawn_lattice", mn, mx, float(default_radius), int(max_count), prec, C.byref(n), None)
    out = np.empty((n.value, 3), dt)
    call("lhi_scene_spawn_lattice", mn, mx, float(default_radius), int(max_count), prec, C.byref(n), _ptr(out))
    return out


def seed_particles(grid, boundary_nodes, prims, seed, precision="fp32"):
    """Seeded 8-per-cell particles (lhi_scene_seed_particles)."""
    prec = PRECISIONS[precision]
    dt = np.float64 if prec == abi.PRECISION_FP64 else np.float32
    nodes = abi.boundary_array(boundary_nodes)
    fp = abi.fluid_array(prims)
    n = C.c_int64()
    call("lhi_scene_seed_particles", C.byref(grid), nodes, len(boundary_nodes), 0, fp, len(prims),
         int(seed), prec, C.byref(n), None, None)
    pos = np.empty((n.value, 3), dt)
    vel = np.empty((n.value, 3), dt)
    call("lhi_scene_seed_particles", C.byref(grid), nodes, len(boundary_nodes), 0, fp, len(prims),
         int(seed), prec, C.byref(n), _ptr(pos), _ptr(vel))
    return pos, vel
