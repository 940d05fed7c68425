"""Algorithmic HBM bytes of one liquid step, for the whole-step roofline
that bench.py and the batched form report.

The model counts the bytes each stage must move at least once (inputs read
once, outputs written once), in the layout of this implementation:

* per particle (P): the cell sort (keys read twice, key and index written,
  the cell-order pass over the indices and ids, the positions gathered in
  sorted order), the liquid SDF (positions read), P2G (position, velocity
  and affine read), G2P + advection (position, permutation index and id
  read; state, key, index and id written);
* per cell of the finest grid (C): the clear, the liquid SDF, P2G's
  normalisation and gravity, the velocity update, the extrapolation's passes
  through tempV, the matrix assembly (with the FP64 finest level of the mixed
  mode), the right-hand side and G2P's face velocities;
* per PCG iteration and active cell of the finest level (A): four fused
  sweeps, the restriction, the prolongation, the SpMV and the CG vector
  updates, times 8/7 for the coarser levels.

The figures are per scalar size s (4 for FP32 / mixed)."""


def particle_bytes(P, s=4):
    sort = 4 + 4 + 8 + 8 + 4 + 2 * 3 * s  # keys twice, (key, index), cell order, gather of the positions
    lphi = 3 * s
    p2g = 15 * s
    g2p = 3 * s + 4 + 4 + 15 * s + 4 + 4 + 4
    return (sort + lphi + p2g + g2p) * P


def grid_bytes(C, s=4, extrap_tempv_passes=1):
    clear = (2 + 9) * s                 # pressure, liquid SDF, v / w / tempV of three components
    lphi = s
    normalize = 3 * 3 * s               # v and w read, v written, per component
    velocity_update = 3 * 4 * s         # v, liquidW, pressure pair read, v written
    extrap = 3 * extrap_tempv_passes * (2 * s + 1)
    lhs = s + 3 * s + 4 * s + 1 + 1 + 4 * 8 // 2  # phi, liquidW, diag + 3 couplings, type, mask, FP64 rows (half)
    rhs = 4 * s + 8 // 2
    g2p_faces = 3 * s
    return (clear + lphi + normalize + velocity_update + extrap + lhs + rhs + g2p_faces) * C


def solve_bytes(A, iterations, s=4):
    sweeps = 4 * (7 * s + 1)
    transfers = (7 * s + 1) + (2 * s + s // 8)
    spmv = 6 * s + 1
    cg = 2 * 8 + 5 * s + 3 * s      # x in FP64 read and written; p, r, Ap, z; p updated
    return iterations * A * (sweeps + transfers + spmv + cg) * 8 / 7


def step_bytes(P, C, A, iterations, s=4):
    """Algorithmic bytes of one step (see the module docstring)."""
    return particle_bytes(P, s) + grid_bytes(C, s) + solve_bytes(A, iterations, s)


def hbm_peak():
    """(GB/s, "measured" | "fallback"): hbm_gbs of MEASURED_PEAKS.json at the
    repository root when present, else 6650 GB/s, an earlier copy-bandwidth
    measurement on the same B200s."""
    import json
    import os
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f).get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"
