"""The batched form: independent scenes stepped concurrently with
asynchronous handles give the same results as stepping them one by one (up
to the summation order of P2G's atomic adds), and the logged training
snapshots have the scene's shapes."""
import numpy as np
import pytest

from liquidhairinteration_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _specs(k, seed=5):
    rng = np.random.default_rng(seed)
    return [scenes.random_scene(rng, n=int(rng.choice([32, 48]))) for _ in range(k)]


def test_async_batch_matches_sequential(lhi):
    from liquidhairinteration_b200.batch import BatchRunner
    specs = _specs(4)
    runner = BatchRunner(specs, "mixed", tune=False)
    seq = [scenes.build(s, "mixed", s.solver_params(num_pre_smooth=2, num_post_smooth=2, coarse_cells=4096,
                                                    coarse_operator=abi.COARSE_GALERKIN))
           for s in specs]
    for _ in range(3):
        st_b = runner.step()
        for s, m in zip(specs, seq):
            m.PreStep(s.dt)
            m.Step(s.dt)
        for k, m in enumerate(seq):
            st = m.GetSolver().Stats()
            assert st["status"] == st_b[k]["status"] == abi.LHI_OK
            assert abs(st["iterations"] - st_b[k]["iterations"]) <= 1
    for k, m in enumerate(seq):
        a = runner.models[k].GetParticleSystem().GetPositions()
        b = m.GetParticleSystem().GetPositions()
        assert np.abs(a - b).max() < 1e-3 / specs[k].n, (k, np.abs(a - b).max())
        m.close()
    runner.close()


def test_batch_logs_training_snapshots(lhi, tmp_path):
    from liquidhairinteration_b200.batch import BatchRunner
    specs = _specs(2, seed=9)
    runner = BatchRunner(specs, "mixed", tune=False, log_dir=str(tmp_path))
    runner.step()
    runner.close()
    shard = np.load(tmp_path / "step0000.npz")
    for k, s in enumerate(specs):
        r = shard[f"r{k}"]
        assert r.shape[1] == s.n ** 3 and r.shape[0] >= 2
        assert shard[f"x{k}"].shape == (s.n ** 3,)
        assert shard[f"fluid{k}"].sum() > 0
        assert np.all(r[:, shard[f"fluid{k}"] == 0] == 0)
