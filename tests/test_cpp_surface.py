"""The C++ host surface (include/lhi_liquid.hpp): LiquidModel<3>, CGSolver<3>
and ParticleSystem<3> over the C-ABI, driven by the reference's frame loop
(tests/cpp/scene_loop.cpp)."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")


def _build():
    subprocess.run(["make", "-s", "-C", CPP], check=True)
    return os.path.join(CPP, "scene_loop")


def test_cpp_surface_compiles(lhi):
    assert os.path.exists(_build())


@pytest.mark.gpu
def test_cpp_scene_loop_runs_on_gpu(lhi):
    exe = _build()
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    res = json.loads(out.stdout.strip().splitlines()[-1])
    print(res)
    assert res["particles"] > 10000
    assert res["correct_volume_moved"] > 0
    assert 0.0 < res["ymin"] < res["ymax"] < 0.6
