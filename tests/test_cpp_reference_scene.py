"""The drop-in under the reference's own Scene<3>.

tests/cpp/ref_scene builds the reference's Scene.cpp, unchanged from the
reference tree, with a binding header in front of the include path: its
"LiquidModel.h" is the B200 liquid step (include/lhi_liquid.hpp), so
Scene<3>'s own constructor (Scene.cpp:13-20) creates the GPU model from the
scene's parameters and hands it its OperatorBoundary<3> through
SetBoundary(BaseBoundary<3>*).  The driver then runs the reference's frame
loop (main.cpp: Init, then PreStep / Step / PostStep with dt = GetCFL()).

CPU: the binary builds where the reference tree is present (it is built
ahead of time for machines without one).  GPU: its particle positions after
Init and 3 steps match the reference's own LiquidModel<3> (the reference
build, oracle/_ref/libref.so) run with the same dt sequence.
"""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import REFERENCE_TREE, ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "ref_scene")
EXE = os.path.join(SRC, "_out", "ref_scene_loop")


def _built(lhi):
    if os.path.isdir(REFERENCE_TREE):
        subprocess.run(["make", "-s", "-C", SRC], check=True, stdout=subprocess.DEVNULL)
    if not os.path.exists(EXE):
        pytest.skip("ref_scene_loop needs the reference tree to build, and no prebuilt binary is present")
    return EXE


def test_reference_scene_builds_against_the_drop_in(lhi):
    exe = _built(lhi)
    syms = subprocess.run(["nm", "-C", exe], capture_output=True, text=True).stdout
    # the reference's Scene<3> constructs the drop-in and binds its boundary object
    assert "lhi_b200::LiquidModel<3>::LiquidModel<Scene<3>" in syms
    assert "SetBoundary<OperatorBoundary<3>" in syms


@pytest.mark.gpu
def test_reference_scene_loop_matches_reference_model(reference_mod, lhi):
    exe = _built(lhi)
    po = reference_mod
    cfg = json.load(open(os.path.join(ROOT, "tests", "golden", "pure_liquid3d.json")))
    cfg["gridDimension"] = [32, 32, 32]
    steps = 3
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "scene.json")
        with open(path, "w") as f:
            json.dump(cfg, f)
        out = os.path.join(d, "pos.bin")
        r = subprocess.run([exe, path, str(steps), out], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
        res = json.loads(r.stdout.strip().splitlines()[-1])
        pos_gpu = np.fromfile(out, np.float32).reshape(-1, 3)
    assert res["spawned"] == res["particles"] == pos_gpu.shape[0] > 0
    ref = po.Reference(cfg)
    ref.init()
    assert ref.num_particles() == pos_gpu.shape[0]
    for dt in res["dt"]:
        dt = np.float32(dt)
        ref.pre_step(dt)
        ref.step(dt)
        ref.post_step(dt)
    pos_ref = ref.get_particles()[0]
    dx = (cfg["maxCoord"][0] - cfg["minCoord"][0]) / cfg["gridDimension"][0]
    d = np.abs(pos_gpu - pos_ref).max()
    assert d <= 1e-3 * dx, (d / dx, res)
