"""Particle snapshots: the reference's trajectory text format and a binary
checkpoint for resuming a run.

Trajectory format (ParticleSystem::WriteToFile, ParticleSystem.cpp:67-85,
and the reference's LiquidData.csv): per frame, one line with the particle
count, then one line of the positions' x, y, z values, each followed by a
comma, printed the way std::ostream prints a float by default (six
significant digits, %g style).  ``write_frame`` appends a frame,
``read_frames`` returns every frame of a file.

Checkpoint: the whole particle state (positions, velocities, affine
matrices, in the model's precision) plus the caller's counters (step, time)
in one ``.npz``; loading it back gives the same bits.
"""
import numpy as np


def format_frame(pos):
    """The two lines of one frame, as WriteToFile prints them."""
    pos = np.asarray(pos).reshape(-1, 3)
    return f"{pos.shape[0]}\n" + "".join("%.6g," % float(v) for v in pos.reshape(-1)) + "\n"


def write_frame(path, pos, append=False):
    with open(path, "a" if append else "w") as f:
        f.write(format_frame(pos))


def read_frames(path):
    """Every frame of a trajectory file as an (n, 3) float64 array."""
    frames = []
    with open(path) as f:
        lines = [ln.strip() for ln in f if ln.strip()]
    for k in range(0, len(lines) - 1, 2):
        count = int(lines[k])
        vals = [float(t) for t in lines[k + 1].split(",") if t]
        if len(vals) != 3 * count:
            raise ValueError(f"frame {k // 2}: {count} particles but {len(vals)} values")
        frames.append(np.array(vals, dtype=np.float64).reshape(count, 3))
    return frames


def save_checkpoint(path, pos, vel, affine, meta=None, **counters):
    """Positions (n x 3), velocities (n x 3) and affine matrices (n x 9,
    column-major), the model description ``meta`` (precision, grid dims and
    bounds) and named scalar counters (step, time, ...)."""
    pos, vel, affine = (np.ascontiguousarray(a) for a in (pos, vel, affine))
    if not (pos.shape[0] == vel.shape[0] == affine.shape[0]) or pos.dtype != vel.dtype or pos.dtype != affine.dtype:
        raise ValueError("positions, velocities and affine matrices must have one count and one dtype")
    extra = {"meta_" + k: np.asarray(v) for k, v in (meta or {}).items()}
    np.savez(path, pos=pos.reshape(-1, 3), vel=vel.reshape(-1, 3), affine=affine.reshape(-1, 9), **extra,
             **{"counter_" + k: np.asarray(v) for k, v in counters.items()})


def load_checkpoint(path, meta=None):
    """dict with pos, vel, affine and the saved counters.  With ``meta``,
    every entry it names must equal the one saved (ValueError otherwise)."""
    with np.load(path) as z:
        for k, want in (meta or {}).items():
            if "meta_" + k not in z.files:
                raise ValueError(f"checkpoint {path} does not record {k}")
            got = z["meta_" + k]
            if got.shape != np.shape(want) or not np.array_equal(got, np.asarray(want)):
                raise ValueError(f"checkpoint {path} was saved with {k} = {got.tolist()}, this model has {want}")
        out = {"pos": z["pos"], "vel": z["vel"], "affine": z["affine"]}
        for k in z.files:
            if k.startswith("counter_"):
                out[k[len("counter_"):]] = z[k].item()
    return out
