"""The whole-step byte model (liquidhairinteration_b200/roofline.py) that
bench.py and the batched form divide by their step times: its parts add
up, scale linearly with particles, cells and solver work, and give the 256^3
dam break about 27 GB per step at 14 PCG iterations."""
from liquidhairinteration_b200 import roofline


def test_step_bytes_parts_and_scaling():
    P, C, A, it = 32190944, 256 ** 3, 2208 * 2048, 14.0
    total = roofline.step_bytes(P, C, A, it)
    assert total == roofline.particle_bytes(P) + roofline.grid_bytes(C) + roofline.solve_bytes(A, it)
    assert roofline.particle_bytes(2 * P) == 2 * roofline.particle_bytes(P)
    assert roofline.grid_bytes(2 * C) == 2 * roofline.grid_bytes(C)
    assert abs(roofline.solve_bytes(A, 2 * it) - 2 * roofline.solve_bytes(A, it)) < 1e-3
    assert roofline.step_bytes(P, C, A, it, s=8) > total
    assert 24e9 < total < 30e9


def test_hbm_peak_has_a_value():
    peak, kind = roofline.hbm_peak()
    assert peak > 1000 and kind in ("measured", "fallback")
