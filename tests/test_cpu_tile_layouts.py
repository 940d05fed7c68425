"""Shared-memory layouts of the staged kernels, checked on the CPU: every
address a kernel can form must fall inside the box or tile it means to read.
The layout constants are read from the CUDA sources so the check follows
any change to them.

- Fused red-black sweep (k_rb_fused): the indices of rb_eval for every cell
  of both colour phases lie inside the Z, R/D/CZ, CX, CY and mask boxes.
- TMA SpMV and restriction (k_spmv_tma, k_restrict_tma): every box index a
  thread forms, and the restriction's 8 children per coarse cell.
- Brick convolution (k_conv_brick): for every tap and K step, each 8-row
  core matrix the tensor-core instruction reads (16 along M, 2 along K) lies
  inside the input brick and is the intended brick row of 8 z voxels, and
  each weight core matrix lies inside its tap's tile.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "liquidhairinteration_b200", "csrc")


def _const(path, name):
    src = open(os.path.join(CSRC, path)).read()
    m = re.search(r"\b%s\s*=\s*([0-9 *]+)[;,]" % name, src)
    assert m, name
    return int(eval(m.group(1)))  # products of integer literals only


def test_fused_sweep_indices_inside_boxes():
    zw = _const("k_solver.cu", "kZW")
    mw = _const("k_solver.cu", "kMW")
    z_box, r_box, c_box = 12 * 12 * zw, 10 * 10 * zw, 11 * 10 * zw
    m_box = 10 * 10 * mw

    def cell(lx, ly, lz):
        ri = ((lx + 1) * 10 + (ly + 1)) * zw + (lz + 4)
        zi = ((lx + 2) * 12 + (ly + 2)) * zw + (lz + 4)
        mi = ((lx + 1) * 10 + (ly + 1)) * mw + (lz + 16)
        xi = ((lx + 2) * 10 + (ly + 1)) * zw + (lz + 4)
        yi = ((lx + 1) * 11 + (ly + 2)) * zw + (lz + 4)
        for idx, size in ((ri, r_box), (ri - 1, r_box), (mi, m_box), (xi, c_box), (xi - 10 * zw, c_box),
                          (yi, c_box), (yi - zw, c_box)):
            assert 0 <= idx < size
        for off in (0, 12 * zw, -12 * zw, zw, -zw, 1, -1):
            assert 0 <= zi + off < z_box
        return zi

    for x0, y0, z0 in ((0, 0, 0), (8, 16, 32), (248, 248, 224)):
        # colour 0 on the tile grown by one cell: 10 x 10 rows of 17
        for q in range(100 * 17):
            row, k = divmod(q, 17)
            lx, ly = row // 10 - 1, row % 10 - 1
            lz = ((x0 + lx + y0 + ly + z0 - 1) & 1) - 1 + 2 * k
            assert -1 <= lz <= 32 and (x0 + lx + y0 + ly + z0 + lz) % 2 == 0
            cell(lx, ly, lz)
        # colour 1 on the tile: 8 x 8 rows of 16
        for q in range(64 * 16):
            row, k = q >> 4, q & 15
            lx, ly = row >> 3, row & 7
            lz = ((x0 + lx + y0 + ly + z0 + 1) & 1) + 2 * k
            assert 0 <= lz <= 31 and (x0 + lx + y0 + ly + z0 + lz) % 2 == 1
            cell(lx, ly, lz)
    # the write-out reads the tile's float4s at z offset 4: 16-byte aligned
    for lx in range(8):
        for ly in range(8):
            for c in range(8):
                assert (((lx + 2) * 12 + (ly + 2)) * zw + 4 + 4 * c) % 4 == 0


@pytest.mark.parametrize("cin", [16, 32, 64])
@pytest.mark.parametrize("cout", [16, 32, 64])
def test_brick_convolution_operands_inside_tiles(cin, cout):
    by, bz = _const("k_learned.cu", "kBrY"), _const("k_learned.cu", "kBrZ")
    bx = _const("k_learned.cu", "kBrX")
    plane = bx * by * bz * 16
    limit = _const("k_learned.cu", "kBrickSmemMax")
    kc = cin // 8
    wbytes = cout * cin * 2
    a_base = 27 * wbytes
    brick_end = a_base + kc * plane
    smem = brick_end + 16
    if smem > limit:
        pytest.skip("this layer runs the gathering kernel")
    assert a_base % 16 == 0 and brick_end % 8 == 0  # operands 16-byte, mbarrier 8-byte aligned
    assert smem < (1 << 18)  # 14-bit descriptor address field in 16-byte units
    for tap in range(27):
        dx, dy, dz = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
        at = a_base + (((dx + 1) * by + (dy + 1)) * bz + (dz + 1)) * 16
        bt = tap * wbytes
        for k in range(cin // 16):
            a0 = at + 2 * k * plane
            for g in range(16):  # M groups: output y rows
                for j in range(2):  # K chunks of this step
                    start = a0 + g * bz * 16 + j * plane
                    assert a_base <= start and start + 128 <= brick_end
                    # the 8 rows are brick voxels (dx+1, g+dy+1, dz+1 .. dz+8) of chunk 2k+j
                    vb = (start - a_base - (2 * k + j) * plane) // 16
                    x, rest = divmod(vb, by * bz)
                    y, z = divmod(rest, bz)
                    assert (x, y, z) == (dx + 1, g + dy + 1, dz + 1) and z + 7 < bz
            b0 = bt + k * 256
            for g in range(cout // 8):
                for j in range(2):
                    start = b0 + g * kc * 128 + j * 128
                    assert bt <= start and start + 128 <= bt + wbytes


def test_spmv_and_restriction_indices_inside_boxes():
    """k_spmv_tma and k_restrict_tma: thread (warp wp = x, lane = z) and row
    ly of a tile read p / z (grown by one cell, z from z0 - 4), diag, the
    coefficients with the -x / -y / -z faces and the mask; the restriction's
    coarse cells read their 8 children from the residual tile."""
    p_box = _const("k_solver.cu", "kP")
    d_box = _const("k_solver.cu", "kD")
    cx_box, cy_box, cz_box = (_const("k_solver.cu", n) for n in ("kCX", "kCY", "kCZ"))
    assert (p_box, d_box, cx_box, cy_box, cz_box) == (10 * 10 * 40, 8 * 8 * 32, 9 * 8 * 32, 8 * 9 * 32, 8 * 8 * 36)
    for wp in range(8):
        for ly in range(8):
            for lane in range(32):
                pi = ((wp + 1) * 10 + (ly + 1)) * 40 + (lane + 4)
                ci = (wp * 8 + ly) * 32 + lane
                for off in (0, 400, -400, 40, -40, 1, -1):
                    assert 0 <= pi + off < p_box
                assert 0 <= ci < d_box and 0 <= ci + 256 < cx_box
                assert 0 <= (wp * 9 + ly + 1) * 32 + lane < cy_box and 0 <= (wp * 9 + ly) * 32 + lane < cy_box
                assert 0 <= (wp * 8 + ly) * 36 + lane + 3 and (wp * 8 + ly) * 36 + lane + 4 < cz_box
    seen = set()
    for t in range(256):  # one coarse cell per thread
        i, j, k = t >> 6, (t >> 4) & 3, t & 15
        for c8 in range(8):
            a, b, c = (c8 >> 2) & 1, (c8 >> 1) & 1, c8 & 1
            idx = ((2 * i + a) * 8 + (2 * j + b)) * 32 + 2 * k + c
            assert 0 <= idx < d_box
            seen.add(idx)
    assert len(seen) == d_box  # the 256 coarse cells cover the fine tile exactly once
