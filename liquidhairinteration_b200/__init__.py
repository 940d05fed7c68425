"""B200-native liquid step: a drop-in for the reference's LiquidModel<3> /
CGSolver<3> pair.  The compute path is liblhi.so (hand-written sm_100a
CUDA behind the C-ABI of include/lhi.h); this package is its Python host
mirror.  ``abi`` holds the ABI constants and structs and loads nothing."""
from . import abi  # noqa: F401

__all__ = ["abi", "model", "scenes"]


def __getattr__(name):
    if name in ("model", "scenes"):
        import importlib
        return importlib.import_module(f".{name}", __name__)
    if name in ("LiquidModel", "Scene", "CGSolver", "ParticleSystem", "RectBoundary", "OperatorBoundary",
                "SolidBoundary"):
        from . import model
        return getattr(model, name)
    raise AttributeError(name)
