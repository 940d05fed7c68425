"""Shared-memory layouts of the staged kernels, checked on the CPU: every
address a kernel can form must fall inside the box or tile it means to read.
The layout constants are read from the CUDA sources so the check follows
any change to them.

- Fused red-black sweep, TMA SpMV and TMA restriction: their index
  arithmetic lives in csrc/layouts.cuh, which the kernels call and which a
  host program (tests/cpp/layout_check.cpp) enumerates for every thread and
  work item.
- Brick convolution (k_conv_brick): for every tap and K step, each 8-row
  core matrix the tensor-core instruction reads (16 along M, 2 along K) lies
  inside the input brick and is the intended brick row of 8 z voxels, each
  weight core matrix lies inside its tap's tile, and every TMA box of every
  brick stage lands 128-byte aligned inside its own plane.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "liquidhairinteration_b200", "csrc")


def _const(path, name):
    src = open(os.path.join(CSRC, path)).read()
    m = re.search(r"\b%s\s*=\s*([0-9 *]+)[;,]" % name, src)
    assert m, name
    return int(eval(m.group(1)))  # products of integer literals only


def test_fused_sweep_spmv_restriction_layouts(tmp_path):
    """Builds tests/cpp/layout_check.cpp against csrc/layouts.cuh -- the
    index functions the fused sweep, the TMA SpMV and the TMA restriction
    call -- and runs it: every index of every work item lies in its box, the
    colour phases cover the grown tile's even cells and the tile's odd cells
    once each, the write-out is 16-byte aligned, and the restriction's
    children cover the fine tile once."""
    exe = str(tmp_path / "layout_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC, os.path.join(ROOT, "tests", "cpp", "layout_check.cpp"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert r.stdout.strip().endswith("ok: 0 failures"), r.stdout


def test_box_constants_match_the_kernels():
    """The fused sweep's stage layout is built from the shared constants."""
    src = open(os.path.join(CSRC, "k_solver.cu")).read()
    for name in ("constexpr int kZW = layout::kZW;", "constexpr int kZ = layout::kZBox;",
                 "constexpr int kR = layout::kRBox;", "constexpr int kC = layout::kCBox;",
                 "constexpr int kMW = layout::kMW;", "constexpr int kM = layout::kMBox;",
                 "constexpr int kP = layout::kPBox, kD = layout::kDBox"):
        assert name in src, name


@pytest.mark.parametrize("cin", [16, 32, 64])
@pytest.mark.parametrize("cout", [16, 32, 64])
def test_brick_convolution_operands_inside_tiles(cin, cout):
    by, bz = _const("k_learned.cu", "kBrY"), _const("k_learned.cu", "kBrZ")
    bx = _const("k_learned.cu", "kBrX")
    box = bx * by * bz * 16  # bytes of one TMA box: 8 channels of every brick voxel
    plane = _const("k_learned.cu", "kBrPlane")
    limit = _const("k_learned.cu", "kBrickSmemMax")
    bars = _const("k_learned.cu", "kBrBars")
    assert box <= plane and plane % 128 == 0
    assert bars >= 6 * 8 + 4 + 4  # six mbarriers, the TMEM address slot and the abort flag
    kc = cin // 8
    wbytes = cout * cin * 2
    a_base = 27 * wbytes
    smem1 = a_base + kc * plane + bars
    if smem1 > limit:
        pytest.skip("this layer runs the gathering kernel")
    stages = 2 if a_base + 2 * kc * plane + bars <= limit else 1
    brick_end = a_base + kc * plane  # stage 0; the operand checks below hold for stage 1 shifted by kc planes
    smem = a_base + stages * kc * plane + bars
    assert smem <= limit
    assert a_base % 128 == 0 and (a_base + stages * kc * plane) % 8 == 0  # TMA 128-byte, mbarrier 8-byte aligned
    for st in range(stages):
        for c in range(kc):
            dst = a_base + (st * kc + c) * plane
            assert dst % 128 == 0 and dst + box <= a_base + (st * kc + c + 1) * plane
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
