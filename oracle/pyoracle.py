"""ctypes access to the CPU oracle and to the reference cross-check build.

TEST INFRASTRUCTURE ONLY.  Loaded by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker; never by the product.

* ``Oracle`` wraps ``oracle/liblhi_oracle.so`` (restatement of the reference's
  liquid path, float or double).
* ``Reference`` wraps ``oracle/_ref/libref.so`` (the reference's own sources
  compiled from the reference tree by ``oracle/refbuild/Makefile``), float only.
"""
import ctypes as C
import json
import os
import tempfile

import numpy as np

from liquidhairinteration_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liblhi_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

_vp = C.c_void_p


def _load_oracle():
    lib = C.CDLL(ORACLE_SO)
    lib.lho_create.restype = _vp
    lib.lho_create.argtypes = [C.POINTER(abi.GridDesc), C.POINTER(abi.SolverParams),
                               C.POINTER(abi.LiquidParams), C.c_int32]
    lib.lho_destroy.argtypes = [_vp]
    lib.lho_get_dx.argtypes = [_vp, C.POINTER(C.c_double)]
    lib.lho_set_boundary.argtypes = [_vp, C.POINTER(abi.BoundaryNode), C.c_int32, C.c_int32]
    lib.lho_set_solid_phi.argtypes = [_vp, _vp]
    lib.lho_boundary_eval.argtypes = [C.POINTER(abi.BoundaryNode), C.c_int32, C.c_int32, C.c_int32,
                                      _vp, C.c_int64, _vp]
    lib.lho_set_particles.argtypes = [_vp, C.c_int64, _vp, _vp, _vp]
    lib.lho_get_particles.argtypes = [_vp, _vp, _vp, _vp]
    lib.lho_num_particles.restype = C.c_int64
    lib.lho_num_particles.argtypes = [_vp]
    lib.lho_field_size.argtypes = [_vp, C.c_int32, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    lib.lho_get_field.argtypes = [_vp, C.c_int32, C.c_int32, _vp]
    lib.lho_set_field.argtypes = [_vp, C.c_int32, C.c_int32, _vp]
    for name in ["lho_clear", "lho_compute_liquid_phi", "lho_particle_to_grid", "lho_grid_to_particle",
                 "lho_solver_init", "lho_solver_build_rhs", "lho_solver_apply_preconditioner"]:
        getattr(lib, name).argtypes = [_vp]
    for name in ["lho_apply_gravity", "lho_velocity_update", "lho_advect_particles", "lho_pre_step"]:
        getattr(lib, name).argtypes = [_vp, C.c_double]
    lib.lho_projection.argtypes = [_vp, C.c_double, C.POINTER(abi.SolveStats)]
    lib.lho_extrapolate.argtypes = [_vp, C.c_int32]
    lib.lho_step.argtypes = [_vp, C.c_double, C.c_int32, C.POINTER(abi.SolveStats)]
    lib.lho_correct_volume.argtypes = [_vp, C.c_double]
    lib.lho_compute_divergence.argtypes = [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.lho_get_cfl.argtypes = [_vp, C.POINTER(C.c_double)]
    lib.lho_solver_build_lhs.argtypes = [_vp, C.c_double, C.c_double]
    lib.lho_solver_solve.argtypes = [_vp, C.c_double, C.c_double, C.POINTER(abi.SolveStats)]
    lib.lho_solver_get_ax.argtypes = [_vp, C.c_int32, _vp, _vp]
    lib.lho_cell_keys.argtypes = [_vp, _vp]
    lib.lho_sort_by_cell.argtypes = [_vp, _vp, _vp]
    lib.lho_set_threads.argtypes = [C.c_int32]
    lib.lho_get_threads.restype = C.c_int32
    lib.lho_set_omp_default_threads.argtypes = [C.c_int32]
    lib.lhi_scene_seed_particles.argtypes = [C.POINTER(abi.GridDesc), C.POINTER(abi.BoundaryNode), C.c_int32,
                                             C.c_int32, C.POINTER(abi.FluidPrim), C.c_int32, C.c_uint64,
                                             C.c_int32, C.POINTER(C.c_int64), _vp, _vp]
    lib.lho_render.argtypes = [_vp, C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_float),
                               C.POINTER(abi.RenderParams), _vp, _vp]
    lib.lho_spawn_lattice.restype = C.c_int64
    lib.lho_spawn_lattice.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                      C.c_int64, C.c_int32, _vp]
    return lib


_ORACLE = None
_REF = None


def oracle_lib():
    global _ORACLE
    if _ORACLE is None:
        _ORACLE = _load_oracle()
    return _ORACLE


def reference_available():
    return os.path.exists(REF_SO)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


EXTRAP_JACOBI = 0
EXTRAP_SERIAL = 1


class Oracle:
    """CPU restatement of LiquidModel<3> + CGSolver<3>; dbl selects double."""

    def __init__(self, grid, solver, liquid, dbl=False):
        self.lib = oracle_lib()
        self.dbl = bool(dbl)
        self.dtype = np.float64 if dbl else np.float32
        self.grid, self.solver, self.liquid = grid, solver, liquid
        self.h = self.lib.lho_create(C.byref(grid), C.byref(solver), C.byref(liquid), int(dbl))
        if not self.h:
            raise RuntimeError("lho_create failed")
        self.n = tuple(grid.dim)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lho_destroy(self.h)
            self.h = None

    @property
    def dx(self):
        d = (C.c_double * 3)()
        self.lib.lho_get_dx(self.h, d)
        return tuple(d)

    def set_boundary(self, nodes, root=0):
        arr = abi.boundary_array(nodes)
        self.lib.lho_set_boundary(self.h, arr, len(nodes), root)

    def set_solid_phi(self, phi):
        phi = np.ascontiguousarray(phi, dtype=self.dtype)
        self.lib.lho_set_solid_phi(self.h, _ptr(phi))

    def set_particles(self, pos, vel=None, aff=None):
        pos = np.ascontiguousarray(pos, dtype=self.dtype).reshape(-1, 3)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=self.dtype).reshape(-1, 3)
        aff = None if aff is None else np.ascontiguousarray(aff, dtype=self.dtype).reshape(-1, 9)
        self.lib.lho_set_particles(self.h, pos.shape[0], _ptr(pos), _ptr(vel), _ptr(aff))

    def num_particles(self):
        return int(self.lib.lho_num_particles(self.h))

    def get_particles(self):
        n = self.num_particles()
        pos = np.empty((n, 3), self.dtype)
        vel = np.empty((n, 3), self.dtype)
        aff = np.empty((n, 9), self.dtype)
        self.lib.lho_get_particles(self.h, _ptr(pos), _ptr(vel), _ptr(aff))
        return pos, vel, aff

    def field(self, name, level=0):
        f = abi.FIELD_NAMES[name] if isinstance(name, str) else name
        cnt = C.c_int64()
        eb = C.c_int32()
        rc = self.lib.lho_field_size(self.h, f, level, C.byref(cnt), C.byref(eb))
        if rc:
            raise ValueError(f"bad field {name}")
        dt = np.uint8 if eb.value == 1 else self.dtype
        out = np.empty(cnt.value, dt)
        self.lib.lho_get_field(self.h, f, level, _ptr(out))
        return out

    def set_field(self, name, data, level=0):
        f = abi.FIELD_NAMES[name] if isinstance(name, str) else name
        cnt = C.c_int64()
        eb = C.c_int32()
        self.lib.lho_field_size(self.h, f, level, C.byref(cnt), C.byref(eb))
        dt = np.uint8 if eb.value == 1 else self.dtype
        data = np.ascontiguousarray(data, dtype=dt).reshape(-1)
        assert data.size == cnt.value
        self.lib.lho_set_field(self.h, f, level, _ptr(data))

    # stages
    def clear(self):
        self.lib.lho_clear(self.h)

    def compute_liquid_phi(self):
        self.lib.lho_compute_liquid_phi(self.h)

    def particle_to_grid(self):
        self.lib.lho_particle_to_grid(self.h)

    def apply_gravity(self, dt):
        self.lib.lho_apply_gravity(self.h, dt)

    def velocity_update(self, dt):
        self.lib.lho_velocity_update(self.h, dt)

    def projection(self, dt):
        st = abi.SolveStats()
        self.lib.lho_projection(self.h, dt, C.byref(st))
        return st.as_dict()

    def extrapolate(self, mode=EXTRAP_JACOBI):
        self.lib.lho_extrapolate(self.h, mode)

    def grid_to_particle(self):
        self.lib.lho_grid_to_particle(self.h)

    def advect_particles(self, dt):
        self.lib.lho_advect_particles(self.h, dt)

    def pre_step(self, dt):
        self.lib.lho_pre_step(self.h, dt)

    def step(self, dt, extrap_mode=EXTRAP_JACOBI):
        st = abi.SolveStats()
        self.lib.lho_step(self.h, dt, extrap_mode, C.byref(st))
        return st.as_dict()

    def divergence(self):
        m = C.c_double()
        mx = C.c_double()
        self.lib.lho_compute_divergence(self.h, C.byref(m), C.byref(mx))
        return m.value, mx.value

    def correct_volume(self, dt):
        self.lib.lho_correct_volume(self.h, dt)

    def cfl(self):
        d = C.c_double()
        self.lib.lho_get_cfl(self.h, C.byref(d))
        return d.value

    def solver_init(self):
        self.lib.lho_solver_init(self.h)

    def build_rhs(self):
        self.lib.lho_solver_build_rhs(self.h)

    def build_lhs(self, rho, dt):
        self.lib.lho_solver_build_lhs(self.h, rho, dt)

    def apply_preconditioner(self):
        self.lib.lho_solver_apply_preconditioner(self.h)

    def solve(self, rho, dt):
        st = abi.SolveStats()
        self.lib.lho_solver_solve(self.h, rho, dt, C.byref(st))
        return st.as_dict()

    def get_ax(self, level, x):
        x = np.ascontiguousarray(x, dtype=self.dtype)
        out = np.empty_like(x)
        self.lib.lho_solver_get_ax(self.h, level, _ptr(x), _ptr(out))
        return out

    def cell_keys(self):
        k = np.empty(self.num_particles(), np.int32)
        self.lib.lho_cell_keys(self.h, _ptr(k))
        return k

    def sort_by_cell(self):
        n = self.num_particles()
        ids = np.empty(n, np.int32)
        cs = np.empty(self.n[0] * self.n[1] * self.n[2] + 1, np.int32)
        self.lib.lho_sort_by_cell(self.h, _ptr(ids), _ptr(cs))
        return ids, cs


def set_threads(n):
    """Threads of the oracle's parallel loops (0: every processor).  Results
    do not depend on it."""
    oracle_lib().lho_set_threads(int(n))


def get_threads():
    return int(oracle_lib().lho_get_threads())


def set_reference_threads(n):
    """OpenMP threads of the reference build's own parallel loops (they
    take OpenMP's default, which this sets for the calling thread)."""
    oracle_lib().lho_set_omp_default_threads(int(n))


def seed_scene(spec, precision="fp32"):
    """(positions, velocities) of a scene's seeded particles from the scene
    generator compiled into the oracle library: the same particles as the
    CUDA library's lhi_scene_seed_particles, with no CUDA library loaded."""
    lib = oracle_lib()
    prec = {"fp32": abi.PRECISION_FP32, "mixed": abi.PRECISION_MIXED, "fp64": abi.PRECISION_FP64}[precision]
    dt = np.float64 if precision == "fp64" else np.float32
    grid = spec.grid_desc()
    nodes = abi.boundary_array(spec.boundary)
    prims = abi.fluid_array(spec.prims)
    n = C.c_int64()
    args = (C.byref(grid), nodes, len(spec.boundary), 0, prims, len(spec.prims), int(spec.seed), prec, C.byref(n))
    rc = lib.lhi_scene_seed_particles(*args, None, None)
    if rc:
        raise RuntimeError(f"lhi_scene_seed_particles failed ({rc})")
    pos = np.empty((n.value, 3), dt)
    vel = np.empty((n.value, 3), dt)
    rc = lib.lhi_scene_seed_particles(*args, _ptr(pos), _ptr(vel))
    if rc:
        raise RuntimeError(f"lhi_scene_seed_particles failed ({rc})")
    return pos, vel


def render(pos, min_coord, max_coord, width=480, height=480, point_size=5.0, color=(0, 0, 255, 255),
           background=(255, 255, 255, 255)):
    """(image height x width x 4, ndc n x 3) of LiquidModel<3>::Render restated."""
    lib = oracle_lib()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    mn = (C.c_float * 3)(*min_coord)
    mx = (C.c_float * 3)(*max_coord)
    rp = abi.make_render_params(width, height, point_size, color, background)
    img = np.empty((height, width, 4), np.uint8)
    ndc = np.empty_like(p)
    rc = lib.lho_render(_ptr(p), p.shape[0], mn, mx, C.byref(rp), _ptr(ndc), _ptr(img))
    if rc:
        raise ValueError("lho_render: bad parameters")
    return img, ndc


def spawn_lattice(min_coord, max_coord, default_radius, max_count, dbl=False):
    lib = oracle_lib()
    mn = (C.c_double * 3)(*min_coord)
    mx = (C.c_double * 3)(*max_coord)
    n = lib.lho_spawn_lattice(mn, mx, default_radius, max_count, int(dbl), None)
    out = np.empty((n, 3), np.float64 if dbl else np.float32)
    lib.lho_spawn_lattice(mn, mx, default_radius, max_count, int(dbl), _ptr(out))
    return out


def boundary_eval(nodes, points, dbl=False):
    lib = oracle_lib()
    arr = abi.boundary_array(nodes)
    dt = np.float64 if dbl else np.float32
    pts = np.ascontiguousarray(points, dtype=dt).reshape(-1, 3)
    out = np.empty(pts.shape[0], dt)
    lib.lho_boundary_eval(arr, len(nodes), 0, int(dbl), _ptr(pts), pts.shape[0], _ptr(out))
    return out


# ---------------------------------------------------------------- reference
def _load_ref():
    lib = C.CDLL(REF_SO)
    lib.ref_create.restype = _vp
    lib.ref_create.argtypes = [C.c_char_p]
    lib.ref_destroy.argtypes = [_vp]
    lib.ref_get_dx.argtypes = [_vp, C.POINTER(C.c_double)]
    lib.ref_init.argtypes = [_vp]
    lib.ref_set_boundary.argtypes = [_vp, C.POINTER(abi.BoundaryNode), C.c_int32, C.c_int32]
    lib.ref_compute_solid_phi.argtypes = [_vp]
    lib.ref_set_particles.argtypes = [_vp, C.c_int64, _vp, _vp, _vp]
    lib.ref_num_particles.restype = C.c_int64
    lib.ref_num_particles.argtypes = [_vp]
    lib.ref_get_particles.argtypes = [_vp, _vp, _vp, _vp]
    lib.ref_get_radius.argtypes = [_vp, _vp]
    lib.ref_get_field.argtypes = [_vp, C.c_int32, C.c_int32, _vp]
    lib.ref_set_field.argtypes = [_vp, C.c_int32, C.c_int32, _vp]
    for name in ["ref_clear", "ref_compute_liquid_phi", "ref_particle_to_grid", "ref_extrapolate",
                 "ref_grid_to_particle", "ref_solver_init", "ref_solver_build_rhs",
                 "ref_solver_apply_preconditioner"]:
        getattr(lib, name).argtypes = [_vp]
    for name in ["ref_apply_gravity", "ref_solve_pressure", "ref_advect_particles", "ref_pre_step",
                 "ref_step", "ref_post_step"]:
        getattr(lib, name).argtypes = [_vp, C.c_float]
    lib.ref_compute_divergence.restype = C.c_double
    lib.ref_compute_divergence.argtypes = [_vp]
    lib.ref_get_cfl.restype = C.c_double
    lib.ref_get_cfl.argtypes = [_vp]
    lib.ref_solver_build_lhs.argtypes = [_vp, C.c_float, C.c_float]
    lib.ref_solver_solve.argtypes = [_vp, C.c_float, C.c_float]
    lib.ref_solver_get_ax.argtypes = [_vp, C.c_int32, _vp, _vp]
    return lib


def ref_lib():
    global _REF
    if _REF is None:
        _REF = _load_ref()
    return _REF


def scene_json(dim, min_coord, max_coord, solver, liquid, dt=0.01, num_particles=0):
    """A config file in the reference's JSON schema (Config/PureLiquid3D.json)."""
    pre = {abi.PRECOND_NONE: "None", abi.PRECOND_JACOBI: "Jacobi",
           abi.PRECOND_MULTIGRID: "Multigrid"}[solver.preconditioner]
    return {
        "SolverParameter": {
            "maxIterations": solver.max_iterations, "tolerance": solver.tolerance,
            "preconditionerType": pre, "numLevel": solver.num_level,
            "numPreSmooth": solver.num_pre_smooth, "numPostSmooth": solver.num_post_smooth,
            "numFinalSmooth": solver.num_final_smooth, "smoothingFactor": solver.smoothing_factor,
        },
        "LiquidParameter": {"numParticles": num_particles, "viscosity": 0.001,
                            "density": liquid.density, "surfaceTension": 0.0728, "correctCycle": 8},
        "HairParameter": {"radius": 0.05, "youngsModulus": 1e5, "shearModulus": 1e5,
                          "viscosity": 1000.0, "density": 1000.0, "refRotation": 0.0,
                          "accumViscosity": True, "numHair": 0, "numParticles": 0, "info": []},
        "dt": dt, "gravity": liquid.gravity,
        "gridDimension": list(dim), "minCoord": list(min_coord), "maxCoord": list(max_coord),
    }


class Reference:
    """The reference's own LiquidModel<3> (float).  Run with OMP_NUM_THREADS=1."""

    dtype = np.float32

    def __init__(self, config):
        self.lib = ref_lib()
        fd, path = tempfile.mkstemp(suffix=".json")
        with os.fdopen(fd, "w") as f:
            json.dump(config, f)
        self.h = self.lib.ref_create(path.encode())
        os.unlink(path)
        if not self.h:
            raise RuntimeError("ref_create failed")
        d = config["gridDimension"]
        self.n = tuple(d)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    @property
    def dx(self):
        d = (C.c_double * 3)()
        self.lib.ref_get_dx(self.h, d)
        return tuple(d)

    def init(self):
        self.lib.ref_init(self.h)

    def set_boundary(self, nodes, root=0):
        arr = abi.boundary_array(nodes)
        self.lib.ref_set_boundary(self.h, arr, len(nodes), root)

    def set_particles(self, pos, vel=None, aff=None):
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float32).reshape(-1, 3)
        aff = None if aff is None else np.ascontiguousarray(aff, dtype=np.float32).reshape(-1, 9)
        self.lib.ref_set_particles(self.h, pos.shape[0], _ptr(pos), _ptr(vel), _ptr(aff))

    def num_particles(self):
        return int(self.lib.ref_num_particles(self.h))

    def get_particles(self):
        n = self.num_particles()
        pos = np.empty((n, 3), np.float32)
        vel = np.empty((n, 3), np.float32)
        aff = np.empty((n, 9), np.float32)
        self.lib.ref_get_particles(self.h, _ptr(pos), _ptr(vel), _ptr(aff))
        return pos, vel, aff

    def radius(self):
        r = np.empty(self.num_particles(), np.float32)
        self.lib.ref_get_radius(self.h, _ptr(r))
        return r

    def _size(self, f, level):
        nx, ny, nz = (v >> level for v in self.n) if f in (abi.FIELD_R, abi.FIELD_Z, abi.FIELD_ADIAG,
                                                          abi.FIELD_ACOEF) else self.n
        sizes = {
            abi.FIELD_VX: (nx + 1) * ny * nz, abi.FIELD_WX: (nx + 1) * ny * nz,
            abi.FIELD_LIQUID_WX: (nx + 1) * ny * nz, abi.FIELD_TEMP_VX: (nx + 1) * ny * nz,
            abi.FIELD_VY: nx * (ny + 1) * nz, abi.FIELD_WY: nx * (ny + 1) * nz,
            abi.FIELD_LIQUID_WY: nx * (ny + 1) * nz, abi.FIELD_TEMP_VY: nx * (ny + 1) * nz,
            abi.FIELD_VZ: nx * ny * (nz + 1), abi.FIELD_WZ: nx * ny * (nz + 1),
            abi.FIELD_LIQUID_WZ: nx * ny * (nz + 1), abi.FIELD_TEMP_VZ: nx * ny * (nz + 1),
            abi.FIELD_SOLID_PHI: (nx + 1) * (ny + 1) * (nz + 1),
            abi.FIELD_IS_VALID: (nx + 1) * (ny + 1) * (nz + 1),
            abi.FIELD_ACOEF: nx * ny * nz * 6,
        }
        return sizes.get(f, nx * ny * nz)

    def field(self, name, level=0):
        f = abi.FIELD_NAMES[name] if isinstance(name, str) else name
        dt = np.uint8 if f == abi.FIELD_IS_VALID else np.float32
        out = np.empty(self._size(f, level), dt)
        rc = self.lib.ref_get_field(self.h, f, level, _ptr(out))
        if rc:
            raise ValueError(f"bad field {name}")
        return out

    def set_field(self, name, data, level=0):
        f = abi.FIELD_NAMES[name] if isinstance(name, str) else name
        dt = np.uint8 if f == abi.FIELD_IS_VALID else np.float32
        data = np.ascontiguousarray(data, dtype=dt).reshape(-1)
        assert data.size == self._size(f, level)
        self.lib.ref_set_field(self.h, f, level, _ptr(data))

    def clear(self):
        self.lib.ref_clear(self.h)

    def compute_liquid_phi(self):
        self.lib.ref_compute_liquid_phi(self.h)

    def particle_to_grid(self):
        self.lib.ref_particle_to_grid(self.h)

    def apply_gravity(self, dt):
        self.lib.ref_apply_gravity(self.h, dt)

    def solve_pressure(self, dt):
        self.lib.ref_solve_pressure(self.h, dt)

    def extrapolate(self):
        self.lib.ref_extrapolate(self.h)

    def grid_to_particle(self):
        self.lib.ref_grid_to_particle(self.h)

    def advect_particles(self, dt):
        self.lib.ref_advect_particles(self.h, dt)

    def pre_step(self, dt):
        self.lib.ref_pre_step(self.h, dt)

    def step(self, dt):
        self.lib.ref_step(self.h, dt)

    def post_step(self, dt):
        self.lib.ref_post_step(self.h, dt)

    def divergence(self):
        return self.lib.ref_compute_divergence(self.h)

    def cfl(self):
        return self.lib.ref_get_cfl(self.h)

    def solver_init(self):
        self.lib.ref_solver_init(self.h)

    def build_rhs(self):
        self.lib.ref_solver_build_rhs(self.h)

    def build_lhs(self, rho, dt):
        self.lib.ref_solver_build_lhs(self.h, rho, dt)

    def apply_preconditioner(self):
        self.lib.ref_solver_apply_preconditioner(self.h)

    def solve(self, rho, dt):
        self.lib.ref_solver_solve(self.h, rho, dt)

    def get_ax(self, level, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.empty_like(x)
        self.lib.ref_solver_get_ax(self.h, level, _ptr(x), _ptr(out))
        return out


# ---------------------------------------------------------- network oracle
def _net_lib():
    lib = oracle_lib()
    if not getattr(lib, "_net_ready", False):
        lib.lho_net_num_params.restype = C.c_longlong
        lib.lho_net_forward.argtypes = [_vp, C.POINTER(C.c_int32), _vp, _vp, _vp, C.c_double, _vp]
        lib.lho_net_backward.argtypes = [_vp, C.POINTER(C.c_int32), _vp, _vp, _vp, C.c_double, _vp, _vp]
        lib.lho_net_set_relu.argtypes = [C.c_int32]
        lib._net_ready = True
    return lib


def net_num_params():
    return int(_net_lib().lho_net_num_params())


def net_set_relu(on):
    _net_lib().lho_net_set_relu(1 if on else 0)


def net_forward(params, r, type_, solid=None, scale=0.0):
    """z = M(r) of the learned preconditioner's network (double sums, BF16
    storage points as on the GPU); r, type_, solid are 3D arrays."""
    lib = _net_lib()
    dims = (C.c_int32 * 3)(*r.shape)
    p = np.ascontiguousarray(params, np.float32)
    rr = np.ascontiguousarray(r, np.float32)
    tt = np.ascontiguousarray(type_, np.uint8)
    ss = None if solid is None else np.ascontiguousarray(solid, np.uint8)
    z = np.empty(r.shape, np.float32)
    lib.lho_net_forward(_ptr(p), dims, _ptr(rr), _ptr(tt), _ptr(ss), float(scale), _ptr(z))
    return z


def net_backward(params, r, type_, solid, dz, scale=0.0):
    """Gradient of sum(dz * M(r)) with respect to the packed parameters."""
    lib = _net_lib()
    dims = (C.c_int32 * 3)(*r.shape)
    p = np.ascontiguousarray(params, np.float32)
    rr = np.ascontiguousarray(r, np.float32)
    tt = np.ascontiguousarray(type_, np.uint8)
    ss = None if solid is None else np.ascontiguousarray(solid, np.uint8)
    d = np.ascontiguousarray(dz, np.float32)
    g = np.empty(p.size, np.float32)
    lib.lho_net_backward(_ptr(p), dims, _ptr(rr), _ptr(tt), _ptr(ss), float(scale), _ptr(d), _ptr(g))
    return g
