"""Particle snapshots on the CPU: the trajectory writer prints numbers the
way the reference's own LiquidData.csv does (its first frame's tokens), the
reader returns what was written, and a checkpoint restores the exact bits."""
import json
import os

import numpy as np
import pytest

from liquidhairinteration_b200 import snapshots

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_writer_prints_like_the_reference_fixture():
    gold = json.load(open(os.path.join(GOLDEN, "liquiddata_frame0.json")))
    toks = gold["head"]  # the first 100 particles of frame 0, as the reference printed them
    pos = np.array([float(t) for t in toks]).reshape(-1, 3)
    text = snapshots.format_frame(pos)
    count, values = text.split("\n")[:2]
    assert count == str(len(toks) // 3)
    assert values.split(",")[:-1] == toks and values.endswith(",")


def test_frames_round_trip(tmp_path):
    rng = np.random.default_rng(4)
    a = rng.uniform(-1, 1, (50, 3)).astype(np.float32)
    b = rng.uniform(-1, 1, (7, 3))
    path = tmp_path / "traj.csv"
    snapshots.write_frame(path, a)
    snapshots.write_frame(path, b, append=True)
    frames = snapshots.read_frames(path)
    assert [f.shape for f in frames] == [(50, 3), (7, 3)]
    for got, want in zip(frames, (a, b)):
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6)  # six significant digits


def test_reader_rejects_a_short_frame(tmp_path):
    path = tmp_path / "bad.csv"
    path.write_text("2\n0.1,0.2,0.3,\n")
    with pytest.raises(ValueError):
        snapshots.read_frames(path)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_checkpoint_restores_exact_bits(tmp_path, dtype):
    rng = np.random.default_rng(5)
    pos, vel, aff = (rng.standard_normal((33, k)).astype(dtype) for k in (3, 3, 9))
    path = tmp_path / "ck.npz"
    snapshots.save_checkpoint(path, pos, vel, aff, step=17, time=0.0354)
    c = snapshots.load_checkpoint(path)
    for k, want in (("pos", pos), ("vel", vel), ("affine", aff)):
        assert c[k].dtype == dtype and np.array_equal(c[k].view(np.uint8), want.view(np.uint8))
    assert c["step"] == 17 and c["time"] == 0.0354


def test_checkpoint_meta_mismatch_rejected(tmp_path):
    pos = np.zeros((4, 3), np.float32)
    aff = np.zeros((4, 9), np.float32)
    meta = {"precision": "fp32", "grid_dim": [16, 16, 16], "min_coord": [0.0] * 3, "max_coord": [1.0] * 3}
    path = tmp_path / "ck.npz"
    snapshots.save_checkpoint(path, pos, pos, aff, meta=meta, step=3)
    assert snapshots.load_checkpoint(path, meta=meta)["step"] == 3
    for k, v in (("precision", "fp64"), ("grid_dim", [16, 16, 32]), ("max_coord", [2.0, 1.0, 1.0])):
        with pytest.raises(ValueError, match=k):
            snapshots.load_checkpoint(path, meta=dict(meta, **{k: v}))
    old = tmp_path / "old.npz"
    snapshots.save_checkpoint(old, pos, pos, aff)
    with pytest.raises(ValueError, match="does not record"):
        snapshots.load_checkpoint(old, meta=meta)


def test_render_oracle_pixel_rule(oracle_mod):
    """The oracle's point rasterisation on a 16 x 16 image with 5-pixel
    points: a point at the domain centre covers pixels 5..9 on both axes, a
    point on the min corner the 2 x 2 pixels it overlaps, and a point beyond
    the max face is clipped."""
    import numpy as np
    pos = np.array([[0.5, 0.5, 0.5], [0.0, 0.0, 0.0], [1.2, 0.5, 0.5]], np.float32)
    img, ndc = oracle_mod.render(pos, (0, 0, 0), (1, 1, 1), 16, 16, 5.0)
    assert np.array_equal(ndc[:2], [[0, 0, 0], [-1, -1, -1]])
    covered = img[..., 0] == 0
    want = np.zeros((16, 16), bool)
    want[5:10, 5:10] = True
    want[0:2, 0:2] = True
    assert np.array_equal(covered, want)
    assert (img[covered] == [0, 0, 255, 255]).all() and (img[~covered] == 255).all()
