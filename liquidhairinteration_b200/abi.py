"""ctypes mirror of include/lhi.h: status codes, constants and POD structs.

Pure data definitions; loading the shared library lives in ``_lib.py``.
"""
import ctypes as C

LHI_OK = 0
LHI_E_INVALID_ARG = 1
LHI_E_CUDA = 2
LHI_E_OOM = 3
LHI_E_NOT_CONVERGED = 4
LHI_E_TIMEOUT = 5
LHI_E_NAN = 6
LHI_E_UNSUPPORTED = 7

STATUS_NAMES = {
    LHI_OK: "LHI_OK",
    LHI_E_INVALID_ARG: "LHI_E_INVALID_ARG",
    LHI_E_CUDA: "LHI_E_CUDA",
    LHI_E_OOM: "LHI_E_OOM",
    LHI_E_NOT_CONVERGED: "LHI_E_NOT_CONVERGED",
    LHI_E_TIMEOUT: "LHI_E_TIMEOUT",
    LHI_E_NAN: "LHI_E_NAN",
    LHI_E_UNSUPPORTED: "LHI_E_UNSUPPORTED",
}

PRECISION_FP32 = 0
PRECISION_MIXED = 1
PRECISION_FP64 = 2

PRECOND_NONE = 0
PRECOND_JACOBI = 1
PRECOND_MULTIGRID = 2
PRECOND_LEARNED = 3

TOL_ABSOLUTE = 0
TOL_RELATIVE = 1

CG_REFERENCE = 0
CG_FLEXIBLE = 1

REGION_INTERIOR = 0
REGION_FLUID = 1

SMOOTHER_REFERENCE = 0
SMOOTHER_DAMPED_GS = 1
SWEEP_FUSED = 0
SWEEP_SPLIT = 1
COARSE_REFERENCE = 0
COARSE_GALERKIN = 1
GUESS_ZERO = 0
GUESS_PREVIOUS = 1

BOUNDARY_RECT = 0
BOUNDARY_SOLID = 1
BOUNDARY_UNION = 2
BOUNDARY_INTERSECTION = 3
BOUNDARY_SUBTRACT = 4
BOUNDARY_NONE = 5

FLUID_BOX = 0
FLUID_SPHERE = 1

FIELD_VX = 0
FIELD_VY = 1
FIELD_VZ = 2
FIELD_WX = 3
FIELD_WY = 4
FIELD_WZ = 5
FIELD_LIQUID_WX = 6
FIELD_LIQUID_WY = 7
FIELD_LIQUID_WZ = 8
FIELD_TEMP_VX = 9
FIELD_TEMP_VY = 10
FIELD_TEMP_VZ = 11
FIELD_PRESSURE = 12
FIELD_LIQUID_PHI = 13
FIELD_SOLID_PHI = 14
FIELD_IS_VALID = 15
FIELD_RHS = 16
FIELD_X = 17
FIELD_P = 18
FIELD_R = 19
FIELD_Z = 20
FIELD_ADIAG = 21
FIELD_ACOEF = 22
FIELD_CELL_KEY = 23
FIELD_PARTICLE_ID = 24
FIELD_CELL_START = 25
FIELD_AP = 26

KERNEL_CATEGORIES = ["sort", "liquid_phi", "p2g", "g2p", "extrapolate", "grid", "lhs", "smooth_fine",
                     "smooth_coarse", "restrict", "prolong", "spmv", "cg_vector"]

FIELD_NAMES = {
    "vx": FIELD_VX, "vy": FIELD_VY, "vz": FIELD_VZ,
    "wx": FIELD_WX, "wy": FIELD_WY, "wz": FIELD_WZ,
    "liquidWx": FIELD_LIQUID_WX, "liquidWy": FIELD_LIQUID_WY, "liquidWz": FIELD_LIQUID_WZ,
    "tempVx": FIELD_TEMP_VX, "tempVy": FIELD_TEMP_VY, "tempVz": FIELD_TEMP_VZ,
    "pressure": FIELD_PRESSURE, "liquidPhi": FIELD_LIQUID_PHI, "solidPhi": FIELD_SOLID_PHI,
    "isValid": FIELD_IS_VALID, "rhs": FIELD_RHS, "x": FIELD_X, "p": FIELD_P,
    "r": FIELD_R, "z": FIELD_Z, "Adiag": FIELD_ADIAG, "Acoef": FIELD_ACOEF,
    "cell_key": FIELD_CELL_KEY, "particle_id": FIELD_PARTICLE_ID, "cell_start": FIELD_CELL_START,
    "Ap": FIELD_AP,
}


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("point_size", C.c_float),
                ("color", C.c_uint8 * 4), ("background", C.c_uint8 * 4)]


def make_render_params(width=480, height=480, point_size=5.0, color=(0, 0, 255, 255),
                       background=(255, 255, 255, 255)):
    """The reference's defaults: a 480 x 480 window (main.cpp:11), white
    background (main.cpp:12), blue points of 5 pixels (LiquidModel.cpp:1140-1149)."""
    return RenderParams(int(width), int(height), float(point_size), (C.c_uint8 * 4)(*color),
                        (C.c_uint8 * 4)(*background))


class GridDesc(C.Structure):
    _fields_ = [("dim", C.c_int32 * 3), ("reserved", C.c_int32),
                ("min_coord", C.c_double * 3), ("max_coord", C.c_double * 3)]


class SolverParams(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("preconditioner", C.c_int32),
                ("tolerance", C.c_double), ("num_level", C.c_int32),
                ("num_pre_smooth", C.c_int32), ("num_post_smooth", C.c_int32),
                ("num_final_smooth", C.c_int32), ("smoothing_factor", C.c_double),
                ("tolerance_mode", C.c_int32), ("cg_variant", C.c_int32),
                ("true_residual_every", C.c_int32), ("update_region", C.c_int32),
                ("smoother", C.c_int32), ("coarse_cells", C.c_int32), ("eager", C.c_int32),
                ("sweep_kernel", C.c_int32), ("coarse_operator", C.c_int32),
                ("initial_guess", C.c_int32)]


class LiquidParams(C.Structure):
    _fields_ = [("density", C.c_double), ("gravity", C.c_double),
                ("particle_radius", C.c_double), ("extrapolate_iterations", C.c_int32),
                ("correct_volume", C.c_int32), ("correct_cycle", C.c_int32), ("reserved", C.c_int32 * 5)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("status", C.c_int32),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("true_residual", C.c_double), ("solve_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BoundaryNode(C.Structure):
    _fields_ = [("kind", C.c_int32), ("use_inside", C.c_int32), ("left", C.c_int32),
                ("right", C.c_int32), ("center", C.c_double * 3), ("half_extent", C.c_double * 3)]


class FluidPrim(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("a", C.c_double * 3),
                ("b", C.c_double * 3), ("velocity", C.c_double * 3)]


def make_grid_desc(dim, min_coord, max_coord):
    g = GridDesc()
    for i in range(3):
        g.dim[i] = int(dim[i])
        g.min_coord[i] = float(min_coord[i])
        g.max_coord[i] = float(max_coord[i])
    return g


def make_solver_params(max_iterations=100, tolerance=1e-5, preconditioner=PRECOND_MULTIGRID,
                       num_level=4, num_pre_smooth=5, num_post_smooth=5, num_final_smooth=20,
                       smoothing_factor=0.5, tolerance_mode=TOL_ABSOLUTE, cg_variant=CG_REFERENCE,
                       true_residual_every=0, update_region=REGION_INTERIOR, smoother=SMOOTHER_REFERENCE,
                       coarse_cells=0, eager=0, sweep_kernel=0, coarse_operator=0, initial_guess=0):
    s = SolverParams()
    s.max_iterations = int(max_iterations)
    s.tolerance = float(tolerance)
    s.preconditioner = int(preconditioner)
    s.num_level = int(num_level)
    s.num_pre_smooth = int(num_pre_smooth)
    s.num_post_smooth = int(num_post_smooth)
    s.num_final_smooth = int(num_final_smooth)
    s.smoothing_factor = float(smoothing_factor)
    s.tolerance_mode = int(tolerance_mode)
    s.cg_variant = int(cg_variant)
    s.true_residual_every = int(true_residual_every)
    s.update_region = int(update_region)
    s.smoother = int(smoother)
    s.coarse_cells = int(coarse_cells)
    s.eager = int(eager)
    s.sweep_kernel = int(sweep_kernel)
    s.coarse_operator = int(coarse_operator)
    s.initial_guess = int(initial_guess)
    return s


def make_liquid_params(density=1000.0, gravity=-9.81, particle_radius=0.0, extrapolate_iterations=5,
                       correct_volume=0, correct_cycle=8):
    p = LiquidParams()
    p.density = float(density)
    p.gravity = float(gravity)
    p.particle_radius = float(particle_radius)
    p.extrapolate_iterations = int(extrapolate_iterations)
    p.correct_volume = int(correct_volume)
    p.correct_cycle = int(correct_cycle)
    return p


def boundary_array(nodes):
    """nodes: list of dicts with kind/use_inside/left/right/center/half_extent."""
    arr = (BoundaryNode * max(1, len(nodes)))()
    for i, n in enumerate(nodes):
        arr[i].kind = int(n["kind"])
        arr[i].use_inside = int(n.get("use_inside", 0))
        arr[i].left = int(n.get("left", -1))
        arr[i].right = int(n.get("right", -1))
        for k in range(3):
            arr[i].center[k] = float(n.get("center", (0, 0, 0))[k])
            arr[i].half_extent[k] = float(n.get("half_extent", (0, 0, 0))[k])
    return arr


def fluid_array(prims):
    arr = (FluidPrim * max(1, len(prims)))()
    for i, p in enumerate(prims):
        arr[i].kind = int(p["kind"])
        for k in range(3):
            arr[i].a[k] = float(p["a"][k])
            arr[i].b[k] = float(p["b"][k]) if k < len(p["b"]) else 0.0
            arr[i].velocity[k] = float(p.get("velocity", (0, 0, 0))[k])
    return arr
